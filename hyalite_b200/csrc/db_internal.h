// db_internal.h -- the device-resident database as the runtime translation units see it.
#pragma once

#include <stdint.h>

#include "host_common.h"
#include "scan_kernel.cuh"

namespace hy {

// Launch shapes. Main scan: groups of MAIN_G lanes, MAIN_R query rows per lane. Winner end
// recovery: one full warp per item.
constexpr int MAIN_G = 8;
constexpr int MAIN_R16 = 16;
constexpr int MAIN_R32 = 16;
constexpr int WIN_G = 32;
constexpr int WIN_R = 16;
constexpr int BLOCK = 256;

struct Partition {
    uint32_t n_items = 0;
    uint64_t n_seqs = 0;
    uint64_t total_cols = 0;
    ItemMeta *d_meta = nullptr;
    void *d_res = nullptr;
};

template <class A>
struct ElemSize {
    static constexpr size_t pe = sizeof(typename A::PE);
};

struct QueryPlan {
    int32_t n_passes = 0;
    int32_t vrow0 = 1;
    uint32_t pass_bytes = 0;
};

inline QueryPlan plan(uint64_t qlen, int rpp, uint64_t al, size_t pe) {
    QueryPlan q;
    q.n_passes = (int32_t)((qlen + rpp - 1) / rpp);
    q.vrow0 = (int32_t)qlen - q.n_passes * rpp + 1;
    q.pass_bytes = (uint32_t)((al + 1) * (uint64_t)rpp * pe);
    return q;
}

}  // namespace hy

struct hy_db {
    int device = 0;
    uint64_t n_seqs = 0, mql = 0, max_t = 0, al = 0;
    int32_t go = 0, ge = 0, min_e = 0, max_e = 0;
    int mode = 0, search_type = 0, layout = HY_LAYOUT_GATHERED;
    hy_score_width width = HY_WIDTH_I8;
    hy_backend backend = HY_BACKEND_CUDA;
    int32_t *d_matrix = nullptr;
    hy::Partition p16, p32;
    uint32_t *d_loc = nullptr;
    uint64_t device_bytes = 0;
};

