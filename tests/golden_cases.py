"""Loader for tests/golden/known_answers.json: resolves sequence references to residues."""
import json
import os

from conftest import DATA, parse_fasta

HERE = os.path.dirname(os.path.abspath(__file__))
_cache = {}


def _genome(name):
    if name not in _cache:
        path = {"phix": "phix174_NC_001422.1.fasta", "lambda": "lambda_NC_001416.1.fasta",
                "cr4": "cr4_adapters.fa"}[name]
        _cache[name] = parse_fasta(os.path.join(DATA, path))
    return _cache[name]


def resolve(spec):
    """A literal list of symbols, ["phix", a, b], "cr4:<i>", ["polyA", n], or a list of those
    (concatenated)."""
    if isinstance(spec, str) and spec.startswith("cr4:"):
        return list(_genome("cr4")[int(spec[4:])][1])
    if isinstance(spec, list) and spec and spec[0] in ("phix", "lambda", "polyA"):
        if spec[0] == "polyA":
            return [0] * spec[1]
        seq = _genome(spec[0])[0][1]
        return list(seq[spec[1]:spec[2]])
    if isinstance(spec, list) and spec and isinstance(spec[0], (list, str)) and not isinstance(spec[0], int):
        out = []
        for part in spec:
            out.extend(resolve(part))
        return out
    return list(spec)


def load():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        return json.load(f)
