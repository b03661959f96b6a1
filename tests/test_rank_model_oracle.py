"""The float64 CPU oracle of the learned root network: its analytic gradient
equals central finite differences (so it can judge the GPU kernels')."""
import numpy as np

import rank_model as R

NP = R.H * (R.H + 4) + 1


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    flat = rng.normal(size=NP) * 0.3
    x, y = rng.random(64), rng.random(64)
    _, g = R.loss_and_grad(flat, x, y)
    h = 1e-6
    for k in range(0, NP, 13):
        fp, fm = flat.copy(), flat.copy()
        fp[k] += h
        fm[k] -= h
        num = (R.loss_and_grad(fp, x, y)[0] - R.loss_and_grad(fm, x, y)[0]) / (2 * h)
        assert abs(num - g[k]) < 1e-7 + 1e-5 * abs(g[k]), k


def test_python_mirrors_match_the_c_structs():
    import ctypes as C

    import tree_layouts as T
    import tree_layouts.learned as LL
    assert LL.NPARAMS == NP == 1153
    size = T.lib().tl_debug_struct_size
    assert size(0) == T.VEB_DTYPE.itemsize == 24
    assert size(1) == C.sizeof(LL.RankModel)
    assert size(2) == LL.LEAF_DTYPE.itemsize == 32
    assert size(3) == C.sizeof(LL.TrainConfig)
