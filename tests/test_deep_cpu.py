"""The library's split tree for the deep tasks (sub-period T / (2 deep_num_steps),
init_split_structure_dimer_deep, source/cpp/QJX/QJX/core.cpp:9928-9981) against the oracle."""
import numpy as np

from oracle import oracle_py as O
from tests.helpers import T2PI


def test_library_deep_tree_equals_oracle():
    import os_d_b200 as q

    N, nsub, deep = 10, 3, 8
    H, Hd, L, Ut = q.build_dimer_deep(N, 1.0, 0.5, 1.0, 1.5, 0.1, 1.0, deep, nsub)
    _, _, _, K0, K1 = O.dimer_operators(N, 1.0, 0.5, 1.0, 1.5, 0.1)
    t_head = 0.5 * T2PI / nsub
    assert np.array_equal(Ut[0], O.split_tree(K0, t_head, deep))
    assert np.array_equal(Ut[1], O.split_tree(K1, t_head, deep))
