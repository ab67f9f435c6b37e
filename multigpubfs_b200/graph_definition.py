"""Lossless schema-2 graph contract (the input format of the native BFS).

Same JSON schema, validation codes, canonical JSON and digest as
``multigpubfs/graph_definition.py:1-69`` of the reference, so graph files and
report digests are interchangeable.  Successor evaluation runs on the GPU
(``mgbfs2_successors_i64``); there is no CPU BFS in this package.
"""
from __future__ import annotations

import copy
import hashlib
import json
import math
import numbers

I64_MIN = -(1 << 63)
I64_MAX = (1 << 63) - 1
_KEYS = {"schema", "name", "generator_names", "action", "start", "expected_max_unique_states"}


def _integer(x):
    if type(x) is not int or not I64_MIN <= x <= I64_MAX:
        raise ValueError("GRAPH_INT64_RANGE")
    return x


def _vector(v):
    if not isinstance(v, list):
        raise ValueError("GRAPH_VECTOR")
    return [_integer(x) for x in v]


class GraphDefinition:
    """Permutation (child[i] = state[g[i]]) or int64 matrix (child = M.S, wrapped,
    then % modulo) action on a start state."""

    def __init__(self, value):
        self._data = copy.deepcopy(value)
        self.validate()

    @classmethod
    def permutation(cls, generators, start, *, name="", generator_names=None, expected_max_unique_states=None):
        return cls({"schema": 2, "name": name,
                    "generator_names": generator_names or [str(i) for i in range(len(generators))],
                    "action": {"kind": "permutation", "degree": len(start), "generators": generators},
                    "start": start, "expected_max_unique_states": expected_max_unique_states})

    @classmethod
    def matrix(cls, rows, cols, generators, start, *, name="", generator_names=None, expected_max_unique_states=None):
        return cls({"schema": 2, "name": name,
                    "generator_names": generator_names or [str(i) for i in range(len(generators))],
                    "action": {"kind": "matrix", "rows": rows, "cols": cols,
                               "generators": [{"matrix": list(mx), "modulo": m} for mx, m in generators]},
                    "start": start, "expected_max_unique_states": expected_max_unique_states})

    @classmethod
    def from_dict(cls, value):
        return cls(value)

    @property
    def start(self):
        return copy.deepcopy(self._data["start"])

    @property
    def action(self):
        return copy.deepcopy(self._data["action"])

    @property
    def name(self):
        return self._data["name"]

    @property
    def generator_names(self):
        return list(self._data["generator_names"])

    @property
    def expected_max_unique_states(self):
        return self._data["expected_max_unique_states"]

    @property
    def state_elements(self):
        return len(self._data["start"])

    @property
    def generator_count(self):
        return len(self._data["action"]["generators"])

    def to_dict(self):
        return copy.deepcopy(self._data)

    def to_json(self):
        return json.dumps(self._data, sort_keys=True, separators=(",", ":"), ensure_ascii=True)

    def digest(self):
        """sha256 of the canonical JSON of schema/action/start (name-independent)."""
        semantic = {k: self._data[k] for k in ("schema", "action", "start")}
        return hashlib.sha256(json.dumps(semantic, sort_keys=True, separators=(",", ":")).encode()).hexdigest()

    def validate(self):
        d = self._data
        if not isinstance(d, dict) or set(d) != _KEYS or d["schema"] != 2:
            raise ValueError("GRAPH_SCHEMA")
        if not isinstance(d["name"], str):
            raise ValueError("GRAPH_NAME")
        start = _vector(d["start"])
        a = d["action"]
        if not isinstance(a, dict) or not isinstance(a.get("generators"), list) or not a["generators"]:
            raise ValueError("GRAPH_GENERATORS")
        names = d["generator_names"]
        if not isinstance(names, list) or len(names) != len(a["generators"]) or not all(isinstance(x, str) for x in names):
            raise ValueError("GRAPH_GENERATOR_NAMES")
        bound = d["expected_max_unique_states"]
        if bound is not None and (type(bound) is not int or not 1 <= bound < 1 << 64):
            raise ValueError("GRAPH_ORBIT_BOUND")
        if a.get("kind") == "permutation":
            n = a.get("degree")
            if set(a) != {"kind", "degree", "generators"} or type(n) is not int or not 1 <= n <= 0xFFFFFFFF \
                    or len(start) != n:
                raise ValueError("GRAPH_PERMUTATION_SHAPE")
            expected = list(range(n))
            for g in a["generators"]:
                if _vector(g) != g or sorted(g) != expected:
                    raise ValueError("GRAPH_PERMUTATION_GENERATOR")
        elif a.get("kind") == "matrix":
            n, m = a.get("rows"), a.get("cols")
            if set(a) != {"kind", "rows", "cols", "generators"} or type(n) is not int or type(m) is not int \
                    or min(n, m) < 1 or n * m > 0xFFFFFFFF or len(start) != n * m:
                raise ValueError("GRAPH_MATRIX_SHAPE")
            for g in a["generators"]:
                if not isinstance(g, dict) or set(g) != {"matrix", "modulo"} or len(_vector(g["matrix"])) != n * n:
                    raise ValueError("GRAPH_MATRIX_GENERATOR")
                mod = g["modulo"]
                if type(mod) is not int or (mod != 0 and not 2 <= mod <= 1 << 31):
                    raise ValueError("GRAPH_MATRIX_MODULUS")
        else:
            raise ValueError("GRAPH_ACTION_KIND")
        return self

    def with_start(self, start):
        """The same graph searched from another start state."""
        value = self.to_dict()
        value["start"] = list(start)
        return GraphDefinition(value)

    def inverse_closed(self):
        """True iff the inverse of every generator is also a generator, so the
        graph is undirected and a layer's neighbours lie within one layer of
        it (the premise of the three-layer-bank history).  Rules of
        graph_definition.py:84-108: a permutation's inverse is compared as a
        tuple; a matrix's inverse must compose to the identity on both sides
        under the action's own arithmetic (int64 wrap, then the modulus), all
        generators must share one modulus, a non-power-of-two modulus must
        keep every row product inside int64, and a modular action needs a
        start whose entries are already reduced."""
        action = self._data["action"]
        if action["kind"] == "permutation":
            present = set(map(tuple, action["generators"]))
            return all(_permutation_inverse(g) in present for g in action["generators"])
        return _matrices_inverse_closed(action["rows"], action["generators"], self._data["start"])

    def successor(self, state, generator):
        """One successor, evaluated by the GPU kernel mgbfs2_successors_i64."""
        state = _vector(state)
        if len(state) != self.state_elements or type(generator) is not int or not 0 <= generator < self.generator_count:
            raise ValueError("GRAPH_SUCCESSOR_ARGUMENT")
        from .kernels import successors_i64
        import torch
        children = successors_i64(self, torch.tensor([state], dtype=torch.int64, device="cuda"))
        return [int(x) for x in children[0, generator].tolist()]


def _permutation_inverse(g):
    """Inverse of a permutation in image form: the positions sorted by image."""
    return tuple(sorted(range(len(g)), key=g.__getitem__))


def _wrap64(x):
    """Two's-complement int64 value of an integer."""
    x &= (1 << 64) - 1
    return x - (1 << 64) if x >> 63 else x


def _matrices_inverse_closed(n, generators, start):
    moduli = {g["modulo"] for g in generators}
    if len(moduli) != 1:
        return False
    (mod,) = moduli
    if mod and mod & (mod - 1):
        # With wrap-before-modulus arithmetic a product row whose reduced
        # magnitude could leave int64 no longer acts as a group element.
        for g in generators:
            rows = [g["matrix"][r * n:(r + 1) * n] for r in range(n)]
            if any(sum(abs(v) for v in row) * (mod - 1) > I64_MAX for row in rows):
                return False
    identity = [1 if r == c else 0 for r in range(n) for c in range(n)]

    def product(a, b):
        # The action applied to a matrix state: right operand already reduced.
        b = [v % mod for v in b] if mod else b
        out = [0] * (n * n)
        for r in range(n):
            for c in range(n):
                v = _wrap64(sum(a[r * n + k] * b[k * n + c] for k in range(n)))
                out[r * n + c] = v % mod if mod else v
        return out

    matrices = [g["matrix"] for g in generators]
    for a in matrices:
        if not any(product(a, b) == identity and product(b, a) == identity for b in matrices):
            return False
    return not mod or all(0 <= x < mod for x in start)


def _flatten(value):
    """Labels of a (possibly nested, possibly tensor) state as a flat list of
    int64 values.  Integral floats become ints; booleans, fractions, strings,
    infinities and NaN raise GRAPH_NONINTEGER_SCALAR, values outside int64
    GRAPH_INT64_RANGE (graph_definition.py:118-129)."""
    flat, pending = [], [value]
    while pending:
        item = pending.pop()
        if hasattr(item, "tolist"):
            item = item.tolist()
        if isinstance(item, (list, tuple)):
            pending.extend(reversed(item))
            continue
        flat.append(_label(item))
    return flat


def _label(x):
    if isinstance(x, bool):
        raise ValueError("GRAPH_NONINTEGER_SCALAR")
    if isinstance(x, numbers.Integral):
        return _integer(int(x))
    if isinstance(x, numbers.Real) and math.isfinite(x) and float(x).is_integer():
        return _integer(int(x))
    raise ValueError("GRAPH_NONINTEGER_SCALAR")


def _cayley_definition(obj):
    """The CayleyPy definition behind a graph object (or the object itself)."""
    if hasattr(obj, "generators_type"):
        return obj
    for attribute in ("definition", "graph_def"):
        if hasattr(obj, attribute):
            return getattr(obj, attribute)
    return obj


def _matrix_degree(matrix):
    return int(matrix.shape[0]) if hasattr(matrix, "shape") else len(matrix)


def from_cayleypy(definition):
    """CayleyPy graph or definition -> GraphDefinition, with generators, start,
    name and generator names carried over exactly (the attributes read by
    graph_definition.py:130-143 of the reference)."""
    d = _cayley_definition(definition)
    kind = d.generators_type.name
    start = _flatten(d.central_state)
    labels = {"name": d.name, "generator_names": list(d.generator_names)}
    if kind == "PERMUTATION":
        return GraphDefinition.permutation(list(map(_flatten, d.generators_permutations)), start, **labels)
    if kind == "MATRIX":
        gens = list(d.generators_matrices)
        n = _matrix_degree(gens[0].matrix)
        cols, ragged = divmod(len(start), n)
        if ragged:
            raise ValueError("GRAPH_MATRIX_SHAPE")
        pairs = [(_flatten(g.matrix), int(g.modulo)) for g in gens]
        return GraphDefinition.matrix(n, cols, pairs, start, **labels)
    raise ValueError("GRAPH_ACTION_KIND")
