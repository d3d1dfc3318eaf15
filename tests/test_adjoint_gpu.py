"""Adjoint (VJP) of the reconstruction sweep through the C ABI.

Checked three ways: against forward-mode dual-number differentiation of the
reference formulas (oracle/weno_oracle_ad.cpp) at 1e-9 max-norm relative (1e-8 for WENO3)
error; against central finite differences (unit-norm direction, steps 1e-4
and 1e-6, smooth data, JS and TENO, with and without MP, cells near kinks
held fixed; per-face and marching adjoints) to 1e-6; and with
torch.autograd.gradcheck through a ctypes autograd wrapper.
"""
import numpy as np
import pytest

from gpu_util import from_dev, rel_err, to_dev

pytestmark = pytest.mark.gpu

# Two FP evaluations of the same derivative (reverse mode here, forward-mode
# duals in the oracle) agree to ~1e-10 where the JS weights switch between
# stencils whose beta differ by orders of magnitude (d alpha/d beta = -2 alpha/beta
# amplifies rounding); the bar is 1e-9 of the array's max norm, 1e-8 for
# WENO3, whose two-stencil weights are the most sensitive.
TOL_AD = 1e-9
TOL_AD3 = 1e-8


@pytest.fixture(scope="module")
def wsb():
    import torch
    assert torch.cuda.is_available()
    import wenostandalone_b200 as w
    w.lib()
    return w


def _varying(order, nc, seed):
    from test_parity_gpu import varying_coefficients
    return varying_coefficients(order, nc, seed=seed)


@pytest.mark.parametrize("mp", [False, True])
@pytest.mark.parametrize("scheme", [0, 3])
@pytest.mark.parametrize("order", [3, 5, 7])
@pytest.mark.parametrize("coef_mode", ["varying", "uniform"])
def test_vjp_matches_dual_number_oracle(wsb, oracle_mod, order, scheme, mp, coef_mode):
    from wenostandalone_b200 import api, fields
    if order == 3 and scheme == 3:
        pytest.skip("WENO3 has no TENO weights in the reference (NaN output)")
    m, n, p, nv = 30, 17, 9, 2
    g = wsb.Grid(m, n, p, nv, 6, scheme=scheme)
    vf = fields.smooth_jump_field(m, n, p, nv, 6, seed=21)
    rng = np.random.default_rng(3)
    for d in range(3):
        nc = g.nc(d)
        coefs = _varying(order, nc, 7 + d) if coef_mode == "varying" else fields.uniform_weno_coefficients(order, nc)
        rs = oracle_mod.reshape(vf, m, n, p, 6, d)
        gL = np.asfortranarray(rng.standard_normal(g.face_shape(d)))
        gR = np.asfortranarray(rng.standard_normal(g.face_shape(d)))
        ref = oracle_mod.vjp(rs, coefs, order, gL, gR, scheme=scheme, mp=mp)
        gv = to_dev(np.zeros(rs.shape))
        flags = wsb.F_MP if mp else 0
        if coef_mode == "varying":
            api.vjp(g, d, order, to_dev(rs), tuple(to_dev(c) for c in coefs), to_dev(gL), to_dev(gR), gv, flags=flags)
        else:
            api.vjp(g, d, order, to_dev(rs), coefs, to_dev(gL), to_dev(gR), gv, flags=flags, uniform=True)
        err = rel_err(from_dev(gv, rs.shape), ref)
        assert err <= (TOL_AD3 if order == 3 else TOL_AD), (d, err)


def _scatter_to_vf(oracle_mod, shape_vf, m, n, p, buff, d, g_rs):
    """Transpose of the reshape: add a v_rs_ws-layout array into v_vf layout."""
    idx = np.arange(np.prod(shape_vf), dtype=np.float64).reshape(shape_vf, order="F")
    rs_idx = oracle_mod.reshape(np.asfortranarray(idx), m, n, p, buff, d).ravel(order="F").astype(np.int64)
    out = np.zeros(int(np.prod(shape_vf)))
    np.add.at(out, rs_idx, np.asarray(g_rs).ravel(order="F"))
    return out.reshape(shape_vf, order="F")


@pytest.mark.parametrize("entry", ["arrays", "uniform"])
def test_vjp_folded_accumulates_three_sweeps(wsb, oracle_mod, entry):
    """Folded sweeps read v_vf directly; with ACCUMULATE the x, y and z
    adjoints sum into one gradient of v_vf (per-face coefficient arrays, and
    the face-independent entry, which takes the marching adjoint where the
    face count is even)."""
    import torch
    from wenostandalone_b200 import api, fields
    m, n, p, nv = 21, 14, 11, 2
    g = wsb.Grid(m, n, p, nv, 6)
    vf = fields.smooth_jump_field(m, n, p, nv, 6, seed=5)
    rng = np.random.default_rng(11)
    ref = np.zeros(vf.shape, order="F")
    gv = torch.zeros(vf.size, dtype=torch.float64, device="cuda")
    v = to_dev(vf)
    for d in range(3):
        coefs = fields.uniform_weno_coefficients(5, g.nc(d))
        rs = oracle_mod.reshape(vf, m, n, p, 6, d)
        gL = np.asfortranarray(rng.standard_normal(g.face_shape(d)))
        gR = np.asfortranarray(rng.standard_normal(g.face_shape(d)))
        ref += _scatter_to_vf(oracle_mod, vf.shape, m, n, p, 6, d,
                              oracle_mod.vjp(rs, coefs, 5, gL, gR, mp=True))
        fl = wsb.F_MP | wsb.F_FOLDED | (wsb.F_ACCUMULATE if d > 0 else 0)
        if entry == "uniform":
            api.vjp(g, d, 5, v, coefs, to_dev(gL), to_dev(gR), gv, flags=fl, uniform=True)
        else:
            api.vjp(g, d, 5, v, tuple(to_dev(c) for c in coefs), to_dev(gL), to_dev(gR), gv, flags=fl)
    assert rel_err(from_dev(gv, vf.shape), ref) <= TOL_AD


def _mp_bad_faces(rs, L, R, margin=1e-3):
    """Faces near a limiter kink: a core face is safe when its WENO states lie
    inside the MP bounds (f90:1564-1608) with `margin` to spare on both sides,
    so a perturbation of ~1e-9 per cell keeps the limiter on its pass-through
    branch.  Returns the unsafe faces as a (ns, c1, c2, V) mask."""
    ns = rs.shape[0] - 6
    o = np.arange(3, ns - 3)
    v = {k: rs[o + 3 + k] for k in range(-2, 3)}
    dm1 = v[0] + v[-2] - 2 * v[-1]
    d0 = v[1] + v[-1] - 2 * v[0]
    dp1 = v[2] + v[0] - 2 * v[1]

    def minmod(dl, dr):
        A, B = 4 * dl - dr, 4 * dr - dl
        same = (np.sign(A) == np.sign(B)) & (np.sign(A) == np.sign(dl)) & (np.sign(A) == np.sign(dr))
        mn = np.minimum(np.minimum(np.abs(A), np.abs(dl)), np.minimum(np.abs(B), np.abs(dr)))
        return np.where(same, np.sign(A) * mn, 0.0)

    mA, mB = minmod(dm1, d0), minmod(d0, dp1)
    safe = np.ones(v[0].shape, dtype=bool)
    for side, x in (("L", L[o]), ("R", R[o])):
        if side == "L":
            UL = v[0] - 2 * (v[1] - v[0]); MD = (v[0] + v[-1] - mA) / 2
            LC = v[0] - (v[1] - v[0]) / 2 + 4 / 3 * mB; vn = v[-1]
        else:
            UL = v[0] + 2 * (v[0] - v[-1]); MD = (v[0] + v[1] - mB) / 2
            LC = v[0] + (v[0] - v[-1]) / 2 + 4 / 3 * mA; vn = v[1]
        lo = np.maximum(np.minimum(np.minimum(v[0], vn), MD), np.minimum(np.minimum(v[0], UL), LC))
        hi = np.minimum(np.maximum(np.maximum(v[0], vn), MD), np.maximum(np.maximum(v[0], UL), LC))
        safe &= (x - lo > margin) & (hi - x > margin)
    bad_face = np.zeros((ns,) + rs.shape[1:], dtype=bool)
    bad_face[3:ns - 3] = ~safe
    return bad_face


def _cells_clear_of(bad_face, rs_shape, half_width):
    """Cells outside every bad face's stencil (+-half_width: 2 for WENO5,
    3 for WENO7)."""
    ns = bad_face.shape[0]
    bad_cell = np.zeros(rs_shape, dtype=bool)
    for k in range(-half_width, half_width + 1):
        bad_cell[3 + k:ns + 3 + k] |= bad_face
    return ~bad_cell


def _mp_safe_cells(rs, L, R, margin=1e-3, half_width=2):
    return _cells_clear_of(_mp_bad_faces(rs, L, R, margin), rs.shape, half_width)


# TENO7 is left out: the reference's beta(4) term (f90:1489-1491) outweighs
# every stencil, so its faces and their gradient are identically zero.
FD_CASES = [(o, sc, mp, entry, 1e-4) for (o, sc, mp) in
            [(5, 0, False), (5, 0, True), (7, 0, False), (7, 0, True), (5, 3, False), (5, 3, True)]
            for entry in ("arrays", "uniform")]
# the configuration's own step, on the benchmarked adjoint (WENO5-JS + MP)
FD_CASES += [(5, 0, True, "uniform", 1e-6), (5, 0, True, "arrays", 1e-6)]


@pytest.mark.parametrize("order,scheme,mp,entry,h", FD_CASES)
def test_vjp_central_differences(wsb, oracle_mod, order, scheme, mp, entry, h):
    """<gv, dv> against (F(v+h dv) - F(v-h dv)) . g / 2h along a unit-norm
    direction dv, on the smooth 128^3-cell, v_size=5 input, cotangents
    N(0,1), JS or TENO (teno_CT=1e-5) weights; the adjoint through the
    per-face coefficient arrays (vjp_kernel) and through the face-independent
    entry (for WENO5-JS + MP the marching adjoint, vjp_march_kernel, which
    the bench times).  dv is zero on the cells whose stencils reach a kink:
    MP faces that _mp_bad_faces flags, and TENO faces whose output changes
    when teno_CT moves by a factor of 2 (a stencil within reach of the
    cutoff).  Bar: 1e-6 relative.

    Steps.  h = 1e-4 with dv random: a cell moves by ~h * 3e-4, far inside
    the 1e-3 limiter margin, and the O(h^2) truncation stays near 1e-9.
    h = 1e-6 (the configuration's step): each forward face state carries
    ~1e-16 of rounding, which the difference quotient turns into ~5e-11 per
    face and ~3e-7 after the ~4e7-term dot product with N(0,1) cotangents --
    against |<gv, dv>| ~ 1 for a random dv that would sit at the bar.  So at
    h = 1e-6 dv is the masked mix (gv + random) / norm, whose <gv, dv> is
    ~|gv| / sqrt(2) ~ 3e3: the same rounding is then ~1e-10 relative, and the
    truncation ~1e-12."""
    import torch
    from wenostandalone_b200 import api, fields
    m = 127
    g = wsb.Grid(m, m, m, 5, 6, scheme=scheme)
    vf = fields.sinusoid_shock_field(m, m, m, 5, 6, seed=4, shock=False)
    gen = torch.Generator(device="cuda").manual_seed(8)
    flags = wsb.F_MP if mp else 0
    hw = (order - 1) // 2
    for d in range(3):
        coefs_np = fields.uniform_weno_coefficients(order, g.nc(d))
        coefs = tuple(to_dev(c) for c in coefs_np)
        rs_np = oracle_mod.reshape(vf, m, m, m, 6, d)
        rs = to_dev(rs_np)
        n = int(np.prod(g.face_shape(d)))
        gL = torch.randn(n, generator=gen, device="cuda", dtype=torch.float64)
        gR = torch.randn(n, generator=gen, device="cuda", dtype=torch.float64)
        gv = torch.empty_like(rs)
        if entry == "uniform":
            api.vjp(g, d, order, rs, coefs_np, gL, gR, gv, flags=flags, uniform=True)
        else:
            api.vjp(g, d, order, rs, coefs, gL, gR, gv, flags=flags)
        dv = torch.randn(rs.numel(), generator=gen, device="cuda", dtype=torch.float64)

        def faces(grid):
            Lw = torch.zeros(n, dtype=torch.float64, device="cuda")
            Rw = torch.zeros_like(Lw)
            api.weno(grid, d, order, rs, coefs, Lw, Rw)
            return from_dev(Lw, g.face_shape(d)), from_dev(Rw, g.face_shape(d))

        bad = np.zeros((g.extents(d)[0],) + rs_np.shape[1:], dtype=bool)
        if scheme == 3:
            lo = faces(wsb.Grid(m, m, m, 5, 6, scheme=3, teno_CT=g.teno_CT * 0.5))
            hi = faces(wsb.Grid(m, m, m, 5, 6, scheme=3, teno_CT=g.teno_CT * 2.0))
            bad |= (lo[0] != hi[0]) | (lo[1] != hi[1])
        if mp:
            bad |= _mp_bad_faces(rs_np, *faces(g))
        mask = None
        if scheme == 3 or mp:
            mask = to_dev(_cells_clear_of(bad, rs_np.shape, hw).astype(np.float64))
            assert float(mask.mean()) > 0.3  # most of the smooth field is away from kinks
            dv = dv * mask
        if h < 1e-5:
            gdir = gv * mask if mask is not None else gv.clone()
            dv = dv / torch.linalg.vector_norm(dv) + gdir / torch.linalg.vector_norm(gdir)
        dv = dv / torch.linalg.vector_norm(dv)
        outs = []
        for sgn in (1.0, -1.0):
            L = torch.zeros(n, dtype=torch.float64, device="cuda")
            R = torch.zeros_like(L)
            api.weno(g, d, order, rs + sgn * h * dv, coefs, L, R, flags=flags)
            outs.append(float((L * gL).sum() + (R * gR).sum()))
        fd = (outs[0] - outs[1]) / (2 * h)
        an = float((gv * dv).sum())
        assert abs(fd - an) <= 1e-6 * abs(an), (d, entry, h, fd, an)


def test_autograd_gradcheck_16cubed(wsb):
    """torch.autograd.gradcheck of the wrapped sweep at 16^3 cells, v_size=2."""
    import torch
    from autograd_weno import WenoSweep
    from wenostandalone_b200 import api, fields
    m = 15
    g = wsb.Grid(m, m, m, 2, 6)
    vf = fields.sinusoid_shock_field(m, m, m, 2, 6, seed=1, shock=False)
    for d in range(3):
        coefs = tuple(to_dev(c) for c in fields.uniform_weno_coefficients(5, g.nc(d)))
        v = to_dev(vf)
        rs = torch.empty(int(np.prod(g.rs_shape(d))), dtype=torch.float64, device="cuda")
        api.reshape(g, d, v, rs)
        rs.requires_grad_(True)
        f = lambda x: WenoSweep.apply(x, g, d, 5, coefs, wsb.F_MP)
        assert torch.autograd.gradcheck(f, (rs,), eps=1e-6, atol=1e-6, rtol=1e-4, fast_mode=True)


def test_vjp_rejects_unsupported(wsb):
    import torch
    from wenostandalone_b200 import _lib as L, api, fields
    g = wsb.Grid(7, 7, 7, 1, 6, scheme=1)
    t = torch.zeros(int(np.prod(g.rs_shape(0))), dtype=torch.float64, device="cuda")
    f = torch.zeros(int(np.prod(g.face_shape(0))), dtype=torch.float64, device="cuda")
    coefs = fields.uniform_weno_coefficients(5, g.nc(0))
    with pytest.raises(L.WenoError) as e:
        api.vjp(g, 0, 5, t, coefs, f, f, torch.zeros_like(t), uniform=True)
    assert e.value.code == L.ERR_UNSUPPORTED
