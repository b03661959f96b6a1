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


def test_compiled_root_equals_the_network():
    """Inference evaluates the trained root through its exact piecewise-linear
    form (tl_debug_rank_model_root, the host twin of the kernels' evaluator):
    at most 33 * 33 pieces, and within float rounding of the float64 network
    everywhere on [0, 1], pieces' ends included."""
    import ctypes as C

    import tree_layouts as T
    import tree_layouts.learned as LL
    L = T.lib()
    L.tl_debug_rank_model_root.argtypes = [C.POINTER(LL.RankModel), C.c_void_p, C.c_uint32, C.c_void_p,
                                           C.POINTER(C.c_uint32)]
    rng = np.random.default_rng(11)
    for trial in range(6):
        m = LL.RankModel()
        flat = rng.normal(size=NP) * (0.5 if trial % 2 else 2.0)
        w1, b1, w2, b2, w3, b3 = R.unpack(flat)
        np.ctypeslib.as_array(m.w1)[:] = w1
        np.ctypeslib.as_array(m.b1)[:] = b1
        np.ctypeslib.as_array(m.w2)[:] = w2
        np.ctypeslib.as_array(m.b2)[:] = b2
        np.ctypeslib.as_array(m.w3)[:] = w3
        m.b3 = b3
        flat32 = np.concatenate([w1, b1, w2.reshape(-1), b2, w3, [b3]]).astype(np.float32).astype(np.float64)
        x = np.concatenate([np.linspace(0, 1, 20001), rng.random(20000)]).astype(np.float32)
        out = np.empty_like(x)
        pieces = C.c_uint32()
        assert L.tl_debug_rank_model_root(C.byref(m), x.ctypes.data, len(x), out.ctypes.data, C.byref(pieces)) == 0
        assert 1 <= pieces.value <= 33 * 33
        ref, _ = R.forward(flat32, x.astype(np.float64))
        scale = max(1.0, float(np.abs(ref).max()))
        assert np.abs(out - ref).max() <= 2e-5 * scale, (trial, np.abs(out - ref).max(), scale)
