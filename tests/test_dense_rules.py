"""Host construction of the dense per-node rule form (CPU).

Random rules on random nodes: evaluating every rule from the dense tables
(each node's distinct populations once, one coefficient row per rule) gives
the term-by-term values, and nodes reading too many distinct populations
make the builder decline.
"""

from __future__ import annotations

import numpy as np

from lbm_b200.solver import dense_rule_tables


def random_rules(rng, n_nodes=40, n_slots=300):
    nodes = np.sort(rng.choice(10_000, n_nodes, replace=False))
    rule_nodes, start, key, coeff = [], [0], [], []
    for s in range(n_nodes):
        for _ in range(rng.integers(0, 5)):  # some nodes carry no rule (immersed-boundary or export nodes)
            k = rng.integers(1, 15)
            rule_nodes.append(nodes[s])
            key.extend(rng.choice(n_slots, k))  # repeated slots within a rule are allowed
            coeff.extend(rng.standard_normal(k))
            start.append(len(key))
    return nodes, np.array(rule_nodes), np.array(start), np.array(key), np.array(coeff)


def test_dense_tables_evaluate_like_the_terms():
    rng = np.random.default_rng(0)
    nodes, rule_nodes, start, key, coeff = random_rules(rng)
    values = rng.standard_normal(300)
    tables = dense_rule_tables(nodes, rule_nodes, start, key, coeff, max_terms=64)
    assert tables is not None
    ut_start, ut_key, rule_row, dense, pos = tables
    assert np.all(rule_row % 4 == 0)
    s_of_rule = np.searchsorted(nodes, rule_nodes)
    for r in range(len(rule_nodes)):
        want = float(coeff[start[r]:start[r + 1]] @ values[key[start[r]:start[r + 1]]])
        s = s_of_rule[r]
        n = ut_start[s + 1] - ut_start[s]
        got = float(dense[rule_row[r]:rule_row[r] + n] @ values[ut_key[ut_start[s]:ut_start[s + 1]]])
        assert got == np.float64(want) or abs(got - want) <= 1e-13 * max(1.0, abs(want))
        # the padding of every row is zero
        pad = (n + 3) // 4 * 4
        assert np.all(dense[rule_row[r] + n:rule_row[r] + pad] == 0.0)
    # every node's distinct keys are distinct and cover its rules' keys
    for s in range(nodes.size):
        mine = ut_key[ut_start[s]:ut_start[s + 1]]
        assert len(set(mine.tolist())) == mine.size
        used = set(key[start[r]:start[r + 1]][t] for r in np.flatnonzero(s_of_rule == s)
                   for t in range(start[r + 1] - start[r]))
        assert used == set(mine.tolist())
    assert pos.size == key.size


def test_builder_declines_nodes_with_too_many_distinct_terms():
    rng = np.random.default_rng(1)
    nodes, rule_nodes, start, key, coeff = random_rules(rng)
    assert dense_rule_tables(nodes, rule_nodes, start, key, coeff, max_terms=4) is None
