"""Predicate trees and their flat submission format.

A predicate is a tree of ``Cmp`` / ``In`` / ``And`` / ``Or`` / ``Not`` nodes
over attribute column slots. ``serialize`` flattens one tree exactly like
the engine's ``fv_pred_serialize`` (engine.cpp:1168-1224): nodes in the
pre-order of ``copy_tree`` (engine.cpp:600-622, node 0 is the root),
children and IN values in side arrays addressed by ``child0`` / ``val0``.
``concat`` joins per-query slices and rebases them like ``GpuConcat::build``
(engine.cpp:1232-1282) into the arrays ``fv_gpu_brute_batch`` /
``fv_gpu_graph_batch`` take.

Evaluation semantics (engine.cpp:397-431): NULL values are stored as NaN and
every comparison with NaN is false; ``NE`` is ``v == v and v != c``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from ._lib import (FV_CMP_EQ, FV_CMP_GE, FV_CMP_GT, FV_CMP_LE, FV_CMP_LT, FV_CMP_NE,
                   FV_NODE_AND, FV_NODE_CMP, FV_NODE_IN, FV_NODE_NOT, FV_NODE_OR, NODE_DTYPE,
                   QD_DTYPE, SPAN_DTYPE)

OPS = {"<": FV_CMP_LT, "<=": FV_CMP_LE, "==": FV_CMP_EQ, ">=": FV_CMP_GE, ">": FV_CMP_GT,
       "!=": FV_CMP_NE}


class Pred:
    def __and__(self, other):
        return And(self, other)

    def __or__(self, other):
        return Or(self, other)

    def __invert__(self):
        return Not(self)


@dataclass(frozen=True)
class Cmp(Pred):
    col: int
    op: str
    value: float

    def __post_init__(self):
        if self.op not in OPS:
            raise ValueError(f"unknown comparison {self.op!r}")


@dataclass(frozen=True)
class In(Pred):
    col: int
    values: tuple

    def __init__(self, col, values):
        object.__setattr__(self, "col", col)
        object.__setattr__(self, "values", tuple(float(v) for v in values))


class And(Pred):
    def __init__(self, *children):
        self.children = list(children)

    def __repr__(self):
        return "And(" + ", ".join(map(repr, self.children)) + ")"


class Or(Pred):
    def __init__(self, *children):
        self.children = list(children)

    def __repr__(self):
        return "Or(" + ", ".join(map(repr, self.children)) + ")"


class Not(Pred):
    def __init__(self, child):
        self.children = [child]

    def __repr__(self):
        return f"Not({self.children[0]!r})"


def to_json(p: Optional[Pred]):
    """A JSON-able nested list form of a tree (None = no filter)."""
    if p is None:
        return None
    if isinstance(p, Cmp):
        return ["cmp", p.col, p.op, p.value]
    if isinstance(p, In):
        return ["in", p.col, list(p.values)]
    kind = {And: "and", Or: "or", Not: "not"}[type(p)]
    return [kind] + [to_json(c) for c in p.children]


def from_json(j) -> Optional[Pred]:
    """Inverse of to_json."""
    if j is None:
        return None
    k = j[0]
    if k == "cmp":
        return Cmp(int(j[1]), j[2], float(j[3]))
    if k == "in":
        return In(int(j[1]), j[2])
    kids = [from_json(c) for c in j[1:]]
    if k == "not":
        return Not(kids[0])
    return (And if k == "and" else Or)(*kids)


@dataclass
class Serialized:
    nodes: np.ndarray     # NODE_DTYPE
    children: np.ndarray  # int32
    invals: np.ndarray    # float64


def serialize(p: Pred) -> Serialized:
    """One tree -> flat arrays, node 0 = root (pre-order)."""
    order: List[Pred] = []
    kids: List[List[int]] = []

    def visit(n: Pred) -> int:
        i = len(order)
        order.append(n)
        kids.append([])
        if isinstance(n, (And, Or, Not)):
            ch = [visit(c) for c in n.children]
            kids[i] = ch
        return i

    visit(p)
    nodes = np.zeros(len(order), NODE_DTYPE)
    children: List[int] = []
    invals: List[float] = []
    for i, n in enumerate(order):
        rec = nodes[i]
        rec["child0"] = len(children)
        rec["val0"] = len(invals)
        if isinstance(n, Cmp):
            rec["kind"], rec["col"], rec["op"], rec["value"] = FV_NODE_CMP, n.col, OPS[n.op], n.value
        elif isinstance(n, In):
            rec["kind"], rec["col"], rec["nvalues"] = FV_NODE_IN, n.col, len(n.values)
            invals.extend(n.values)
        else:
            rec["kind"] = {And: FV_NODE_AND, Or: FV_NODE_OR, Not: FV_NODE_NOT}[type(n)]
            rec["nchildren"] = len(kids[i])
            children.extend(kids[i])
    return Serialized(nodes, np.asarray(children, np.int32), np.asarray(invals, np.float64))


@dataclass
class BatchPred:
    """Concatenated, rebased predicate arrays of one batch (GpuConcat)."""
    qd: np.ndarray
    nodes: np.ndarray
    children: np.ndarray
    invals: np.ndarray
    spans: np.ndarray
    spanoff: np.ndarray
    dedup: np.ndarray
    roots: np.ndarray = field(default=None)  # int32 per query (qd.proot)


def concat(preds: Sequence[Optional[Pred]], count: int,
           entries: Optional[Sequence[int]] = None) -> BatchPred:
    nq = len(preds)
    qd = np.zeros(nq, QD_DTYPE)
    node_parts, child_parts, val_parts = [], [], []
    base_n = base_c = base_v = 0
    cache = {}
    for q, p in enumerate(preds):
        if p is None:
            qd[q]["proot"] = -1
        else:
            key = id(p)
            s = cache.get(key)
            if s is None:
                s = cache[key] = serialize(p)
            n = s.nodes.copy()
            n["child0"] += base_c
            n["val0"] += base_v
            node_parts.append(n)
            child_parts.append(s.children + base_n)
            val_parts.append(s.invals)
            qd[q]["proot"] = base_n
            base_n += len(n)
            base_c += len(s.children)
            base_v += len(s.invals)
        qd[q]["need_eval"] = 1
        qd[q]["total"] = count
        if entries is not None:
            qd[q]["entry"] = entries[q]
    nodes = np.concatenate(node_parts) if node_parts else np.zeros(0, NODE_DTYPE)
    children = (np.concatenate(child_parts).astype(np.int32) if child_parts
                else np.zeros(0, np.int32))
    invals = np.concatenate(val_parts) if val_parts else np.zeros(0, np.float64)
    return BatchPred(qd, nodes, children, invals, np.zeros(0, SPAN_DTYPE),
                     np.zeros(0, np.uint64), np.zeros(nq, np.uint8),
                     qd["proot"].astype(np.int32))


def eval_numpy(p: Optional[Pred], cols: np.ndarray) -> np.ndarray:
    """Boolean mask of rows satisfying p; cols is [ncols, N] float64. Used by
    host-side tooling (selectivity estimates, workload construction)."""
    n = cols.shape[1]
    if p is None:
        return np.ones(n, bool)
    with np.errstate(invalid="ignore"):
        if isinstance(p, Cmp):
            v = cols[p.col]
            c = p.value
            return {"<": v < c, "<=": v <= c, "==": v == c, ">=": v >= c, ">": v > c,
                    "!=": (v == v) & (v != c)}[p.op]
        if isinstance(p, In):
            v = cols[p.col]
            m = np.zeros(n, bool)
            for x in p.values:
                m |= v == x
            return m
        if isinstance(p, And):
            m = np.ones(n, bool)
            for c in p.children:
                m &= eval_numpy(c, cols)
            return m
        if isinstance(p, Or):
            m = np.zeros(n, bool)
            for c in p.children:
                m |= eval_numpy(c, cols)
            return m
        if isinstance(p, Not):
            return ~eval_numpy(p.children[0], cols)
    raise TypeError(p)
