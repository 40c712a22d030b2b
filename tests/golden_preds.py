"""Predicate shapes of the golden fixtures (shared by tests/golden/make_golden.py
and the tests that read the fixtures)."""
from paves_b200 import datagen
from paves_b200.pred import And, Cmp, In, Not, Or

P, CAT = datagen.COL_PRICE, datagen.COL_CATEGORY


def brute_predicates():
    return [
        None,
        datagen.config1_predicate(),
        And(Cmp(P, "<", 10.0), Cmp(CAT, "==", 3.0)),
        Cmp(P, "<", 10.0),
        In(CAT, [3]),
        In(CAT, [1, 4, 7]),
        Cmp(P, "<", 700.0),
        Not(In(CAT, [3])),
        Or(Cmp(P, "<", 5.0), Cmp(CAT, "==", 9.0)),
        Cmp(CAT, "!=", 2.0),
        Not(Cmp(P, ">=", 300.0)),        # NULL (NaN) prices pass through NOT
        Cmp(P, "<", -1.0),               # no match
        And(Cmp(P, ">=", 100.0), Cmp(P, "<=", 120.0), In(CAT, [0, 5, 9])),
        Cmp(P, "==", float("nan")),      # always false
    ]


def graph_predicates():
    return [None, In(CAT, [3]), Cmp(P, "<", 50.0), Cmp(P, "<", 500.0)]
