"""Host-side mirror of the reference harness interface over the C ABI.

`Grid` is the &grid_params namelist (wilfonba/WenoStandalone
inputs/weno_standalone.f90:117-118).  `Harness` owns the harness's module
arrays on the GPU (f90:87-100) and exposes its routines under their
reference names: s_initialize_weno_{x,y,z} (f90:281-330),
s_order1_copy_{x,y,z} (f90:332-390), s_weno3_kernel (f90:392-475),
s_weno5_kernel_dispatch / s_weno5_kernel_{x,y,z} (f90:477-1417),
s_weno7_kernel (f90:1419-1542), s_preserve_monotonicity (f90:1544-1615) and
f_checksum (f90:1617-1620).  The module-level functions are the
device-pointer calls (arrays as 1-D CUDA tensors in Fortran element order).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from ._lib import check, lib


@dataclass
class Grid:
    m_cells: int = 199
    n_cells: int = 199
    p_cells: int = 199
    v_size: int = 8
    buff_size: int = 6
    scheme: int = L.JS
    weno_eps: float = 1e-16
    teno_CT: float = 1e-5

    @classmethod
    def from_namelist(cls, m=199, n=199, p=199, v_size=8, buff_size=6, weno_eps=1e-16,
                      wenojs=True, teno_CT=1e-5, teno_enabled=True):
        """The namelist's `wenojs` logical: JS when true; when false the
        harness falls through to TENO (if its compile-time `teno` is on,
        f90:74) or to no weight family at all (alpha = 0, NaN output)."""
        scheme = L.JS if wenojs else (L.TENO if teno_enabled else L.NONE)
        return cls(m, n, p, v_size, buff_size, scheme, weno_eps, teno_CT)

    def c(self) -> L.WenoGrid:
        return L.WenoGrid(self.m_cells, self.n_cells, self.p_cells, self.v_size, self.buff_size,
                          self.scheme, self.weno_eps, self.teno_CT)

    @property
    def N(self):
        b = self.buff_size
        return (self.m_cells + 2 * b + 1, self.n_cells + 2 * b + 1, self.p_cells + 2 * b + 1)

    def extents(self, d: int):
        N1, N2, N3 = self.N
        return {0: (N1, N2, N3), 1: (N2, N1, N3), 2: (N3, N2, N1)}[d]

    def vf_shape(self):
        return tuple(n + 6 for n in self.N) + (self.v_size,)

    def rs_shape(self, d):
        ns, c1, c2 = self.extents(d)
        return (ns + 6, c1, c2, self.v_size)

    def face_shape(self, d):
        ns, c1, c2 = self.extents(d)
        return (ns, c1, c2, self.v_size)

    def nc(self, d):
        return self.extents(d)[0] - 6

    def face_states(self, d, order=5):
        """Reconstructed scalars one sweep writes (vL and vR)."""
        ns, c1, c2 = self.extents(d)
        nf = ns if order == 3 else ns - 6
        return 2 * nf * c1 * c2 * self.v_size


_OFFSETS = (0.03, 0.05, 0.07)  # f90:190-192


class Harness:
    """The harness's module state on one GPU (handle API)."""

    def __init__(self, grid: Grid, precision: int = L.FP64):
        self.grid = grid
        self.precision = precision
        h = ctypes.c_int(0)
        check(lib().weno_sb_init(ctypes.byref(grid.c()), precision, ctypes.byref(h)))
        self.handle = h.value

    # -- data movement (target update to/from) --
    def shape_of(self, which: int):
        g = self.grid
        if which == L.A_V_VF:
            return g.vf_shape()
        k, d = divmod(which - 1, 3)
        nc = g.nc(d)
        return [g.rs_shape(d), g.face_shape(d), g.face_shape(d), (nc, 5, 3), (nc, 5, 3),
                (5, nc), (5, nc), (nc, 5, 6)][k]

    def upload(self, which: int, arr: np.ndarray) -> None:
        a = np.asfortranarray(arr, dtype=np.float64)
        assert a.shape == tuple(self.shape_of(which)), (a.shape, self.shape_of(which))
        check(lib().weno_sb_upload(self.handle, which, a.ctypes.data))

    def upload_async(self, which: int, host) -> None:
        """weno_sb_upload_async from `host` (a page-locked CPU torch tensor
        or a numpy array in the array's Fortran order), kept referenced until
        the next upload: the folded sweeps overlap the copy."""
        if not hasattr(host, "data_ptr"):
            host = np.asfortranarray(host, dtype=np.float64)
        self._pending = host
        ptr = host.data_ptr() if hasattr(host, "data_ptr") else host.ctypes.data
        check(lib().weno_sb_upload_async(self.handle, which, ptr))

    def download(self, which: int) -> np.ndarray:
        out = np.empty(self.shape_of(which), order="F")
        check(lib().weno_sb_download(self.handle, which, out.ctypes.data))
        return out

    def device_ptr(self, which: int) -> int:
        p = ctypes.c_void_p()
        check(lib().weno_sb_array_info(self.handle, which, ctypes.byref(p), None, None))
        return p.value

    def upload_coefficients(self, d: int, coefs) -> None:
        pL, pR, dL, dR, bc = coefs
        self.upload(L.A_POLYL(d), pL)
        self.upload(L.A_POLYR(d), pR)
        self.upload(L.A_DL(d), dL)
        self.upload(L.A_DR(d), dR)
        self.upload(L.A_BETA(d), bc)

    def fill_harness_data(self, field: np.ndarray | None = None) -> None:
        """s_initialize_data's fill + upload (f90:189-203) with the
        harness's synthetic field and coefficients."""
        from . import fields
        g = self.grid
        if field is None:
            field = fields.harness_field(g.m_cells, g.n_cells, g.p_cells, g.v_size, g.buff_size)
        self.upload(L.A_V_VF, field)
        for d in range(3):
            self.upload_coefficients(d, fields.harness_coefficients(g.nc(d), _OFFSETS[d]))

    # -- the reference's routines --
    def s_initialize_weno(self, d: int) -> None:
        check(lib().weno_sb_initialize_weno(self.handle, d))

    def s_initialize_weno_x(self): self.s_initialize_weno(0)
    def s_initialize_weno_y(self): self.s_initialize_weno(1)
    def s_initialize_weno_z(self): self.s_initialize_weno(2)

    def weno(self, d: int, order: int, flags: int = 0) -> None:
        check(lib().weno_sb_weno(self.handle, d, order, flags))

    def s_order1_copy(self, d): self.weno(d, 1)
    def s_weno3_kernel(self, d): self.weno(d, 3)
    def s_weno5_kernel_dispatch(self, d, split=False):
        self.weno(d, 5, L.F_SPLIT if split else 0)
    def s_weno5_kernel_specialized(self, d): self.weno(d, 5, L.F_SPECIALIZED)
    def s_weno7_kernel(self, d): self.weno(d, 7)

    def s_preserve_monotonicity(self, d: int) -> None:
        check(lib().weno_sb_preserve_monotonicity(self.handle, d))

    def checksum(self, which: int) -> float:
        out = ctypes.c_double(0.0)
        check(lib().weno_sb_checksum(self.handle, which, ctypes.byref(out)))
        return out.value

    def sync(self) -> None:
        check(lib().weno_sb_sync(self.handle))

    def close(self) -> None:
        if self.handle:
            check(lib().weno_sb_finalize(self.handle))
            self.handle = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            if self.handle:
                lib().weno_sb_finalize(self.handle)
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Device-pointer API on CUDA tensors (1-D, Fortran element order)
# ---------------------------------------------------------------------------
def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def _stream(stream) -> int:
    if stream is None:
        import torch
        return int(torch.cuda.current_stream().cuda_stream)
    return int(stream)


def _dtype_of(t) -> int:
    import torch
    return L.FP32 if t.dtype == torch.float32 else L.FP64


def _need(name: str, t, n: int, dtypes) -> None:
    """Refuse a tensor the C call would read or write out of its bounds: the
    device-pointer entries take bare pointers, so the element type and count
    are checked here (a float32 array where FP64 is read, or a short array,
    would otherwise make the kernel access memory it does not own)."""
    import torch
    if t is None:
        raise ValueError(f"{name} is missing")
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype not in dtypes:
        raise TypeError(f"{name} has dtype {t.dtype}; expected {' or '.join(str(x) for x in dtypes)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.numel() < n:
        raise ValueError(f"{name} has {t.numel()} elements; the call accesses {n}")


def _f64():
    import torch
    return (torch.float64,)


def _same(t):
    return (t.dtype,) if t is not None else _f64()


def _check_sweep(grid: Grid, d: int, v_in, vL, vR, folded: bool) -> None:
    """Sizes of a sweep's arrays; an invalid direction is left for the
    library to report (WENO_SB_ERR_ARG)."""
    import torch
    if d not in (0, 1, 2):
        return
    _need("vL", vL, int(np.prod(grid.face_shape(d))), (torch.float64, torch.float32))
    _need("vR", vR, int(np.prod(grid.face_shape(d))), _same(vL))
    n_in = int(np.prod(grid.vf_shape() if folded else grid.rs_shape(d)))
    _need("v_in", v_in, n_in, _same(vL))


def reshape(grid: Grid, d: int, v_vf, out, stream=None) -> None:
    import torch
    _need("v_vf", v_vf, int(np.prod(grid.vf_shape())), _f64())
    _need("out", out, int(np.prod(grid.rs_shape(d))), (torch.float64, torch.float32))
    check(lib().weno_sb_reshape_dev(ctypes.byref(grid.c()), d, _dtype_of(out), _ptr(v_vf), _ptr(out),
                                    _stream(stream)))


def order1_copy(grid: Grid, d: int, v_vf, vL, vR, stream=None) -> None:
    import torch
    _need("v_vf", v_vf, int(np.prod(grid.vf_shape())), _f64())
    _need("vL", vL, int(np.prod(grid.face_shape(d))), (torch.float64, torch.float32))
    _need("vR", vR, int(np.prod(grid.face_shape(d))), _same(vL))
    check(lib().weno_sb_order1_dev(ctypes.byref(grid.c()), d, _dtype_of(vL), _ptr(v_vf), _ptr(vL), _ptr(vR),
                                   _stream(stream)))


def coefs_struct(coefs) -> L.WenoCoefs:
    pL, pR, dL, dR, bc = coefs
    return L.WenoCoefs(_ptr(pL), _ptr(pR), _ptr(dL), _ptr(dR), _ptr(bc))


def weno(grid: Grid, d: int, order: int, v_in, coefs, vL, vR, flags: int = 0, stream=None) -> None:
    cs = coefs if isinstance(coefs, L.WenoCoefs) else coefs_struct(coefs)
    if order in (1, 3, 5, 7):
        _check_sweep(grid, d, v_in, vL, vR, bool(flags & L.F_FOLDED))
    check(lib().weno_sb_weno_dev(ctypes.byref(grid.c()), d, order, flags, _dtype_of(vL), _ptr(v_in),
                                 ctypes.byref(cs), _ptr(vL), _ptr(vR), _stream(stream)))


def face_coefs(coefs, face: int = 0) -> L.WenoFaceCoefs:
    """One face's coefficients (from numpy arrays in the harness layouts) as
    the weno_sb_face_coefs struct."""
    pL, pR, dL, dR, bc = (np.asarray(c) for c in coefs)
    f = L.WenoFaceCoefs()
    for s in range(3):
        for r in range(5):
            f.polyL[s][r] = float(pL[face, r, s])
            f.polyR[s][r] = float(pR[face, r, s])
    for r in range(5):
        f.dL[r] = float(dL[r, face])
        f.dR[r] = float(dR[r, face])
    for s in range(6):
        for r in range(5):
            f.beta_coef[s][r] = float(bc[face, r, s])
    return f


def weno_uniform(grid: Grid, d: int, order: int, v_in, face, vL, vR, flags: int = 0, stream=None) -> None:
    """Reconstruction with face-independent coefficients (`face`: a
    WenoFaceCoefs, or numpy coefficient arrays whose face 0 is used)."""
    f = face if isinstance(face, L.WenoFaceCoefs) else face_coefs(face)
    if order in (1, 3, 5, 7):
        _check_sweep(grid, d, v_in, vL, vR, bool(flags & L.F_FOLDED))
    check(lib().weno_sb_weno_uniform_dev(ctypes.byref(grid.c()), d, order, flags, _dtype_of(vL), _ptr(v_in),
                                         ctypes.byref(f), _ptr(vL), _ptr(vR), _stream(stream)))


def vjp(grid: Grid, d: int, order: int, v_in, coefs, gL, gR, gv, flags: int = 0, stream=None,
        uniform: bool = False) -> None:
    """Adjoint of one sweep: gv = (dF/dv)^T (gL, gR).  `coefs`: device
    coefficient tensors (per face), or with uniform=True numpy arrays /
    a WenoFaceCoefs whose face 0 applies to every face."""
    if uniform:
        f = coefs if isinstance(coefs, L.WenoFaceCoefs) else face_coefs(coefs)
        cs, fp = None, ctypes.byref(f)
    else:
        cs = coefs if isinstance(coefs, L.WenoCoefs) else coefs_struct(coefs)
        cs, fp = ctypes.byref(cs), None
    if d in (0, 1, 2) and order in (3, 5, 7):
        n_in = int(np.prod(grid.vf_shape() if flags & L.F_FOLDED else grid.rs_shape(d)))
        _need("v_in", v_in, n_in, _f64())
        _need("gv", gv, n_in, _f64())
        _need("gL", gL, int(np.prod(grid.face_shape(d))), _f64())
        _need("gR", gR, int(np.prod(grid.face_shape(d))), _f64())
    check(lib().weno_sb_vjp_dev(ctypes.byref(grid.c()), d, order, flags, _ptr(v_in), cs, fp, _ptr(gL), _ptr(gR),
                                _ptr(gv), _stream(stream)))


def preserve_monotonicity(grid: Grid, d: int, v_rs_ws, vL, vR, stream=None) -> None:
    _check_sweep(grid, d, v_rs_ws, vL, vR, False)
    check(lib().weno_sb_preserve_monotonicity_dev(ctypes.byref(grid.c()), d, _dtype_of(vL), _ptr(v_rs_ws),
                                                  _ptr(vL), _ptr(vR), _stream(stream)))


def checksum(arr, stream=None) -> float:
    import torch
    scratch = torch.empty(int(lib().weno_sb_checksum_scratch_bytes(arr.numel())) // 8 + 1,
                          dtype=torch.float64, device=arr.device)
    res = torch.empty(1, dtype=torch.float64, device=arr.device)
    check(lib().weno_sb_checksum_dev(_dtype_of(arr), _ptr(arr), arr.numel(), _ptr(scratch), _ptr(res),
                                     _stream(stream)))
    return float(res.item())


class Batch:
    """Many uneven blocks' sweeps in one graph launch (a persistent kernel over
    all blocks, or per-block specialised sweeps on parallel graph branches;
    autotune() picks the faster).

    `entries`: sequence of dicts with keys grid (Grid), dir, order, flags,
    v_in, coefs (5 device tensors), vL, vR (CUDA tensors; float32 tensors
    select FP32-bulk storage)."""

    def __init__(self, entries):
        import torch
        n = len(entries)
        arr = (L.WenoBlock * n)()
        self._keep = []
        for i, e in enumerate(entries):
            b = arr[i]
            b.grid = e["grid"].c()
            b.dir = e["dir"]
            b.order = e["order"]
            b.flags = e.get("flags", 0)
            b.dtype = L.FP32 if e["vL"].dtype == torch.float32 else L.FP64
            b.v_in = _ptr(e["v_in"])
            b.coefs = coefs_struct(e["coefs"])
            b.vL = _ptr(e["vL"])
            b.vR = _ptr(e["vR"])
            self._keep.append(e)
        h = ctypes.c_int(0)
        check(lib().weno_sb_batch_create(arr, n, ctypes.byref(h)))
        self.handle = h.value

    def autotune(self, stream=None):
        t, u, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(lib().weno_sb_batch_autotune(self.handle, _stream(stream), ctypes.byref(t), ctypes.byref(u),
                                           ctypes.byref(ms)))
        return t.value, u.value, ms.value

    def configure(self, mode: int, threads: int = 128, cols_per_item: int = 8, branches: int = 8):
        """mode 0: one persistent kernel (threads x cols_per_item work items);
        mode 1: a graph of per-block specialised sweeps on `branches` branches;
        mode 2: grouped TMA marching sweeps (one launch per kernel instance and
        coefficient set, cols_per_item = faces per work item, 8..4096) on
        `branches` branches, the blocks no group takes as in mode 1."""
        check(lib().weno_sb_batch_configure(self.handle, mode, threads, cols_per_item, branches))

    def query(self):
        """(mode, threads, cols_per_item, branches) of the current choice."""
        v = [ctypes.c_int() for _ in range(4)]
        check(lib().weno_sb_batch_query(self.handle, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def launch(self, stream=None):
        check(lib().weno_sb_batch_launch(self.handle, _stream(stream)))

    def close(self):
        if self.handle:
            check(lib().weno_sb_batch_destroy(self.handle))
            self.handle = 0

    def __del__(self):
        try:
            if self.handle:
                lib().weno_sb_batch_destroy(self.handle)
        except Exception:
            pass


def weno_coefficients(order: int, x_cb):
    """(polyL, polyR, dL, dR, beta_coef) of WENO-JS for order 3/5/7 on the
    grid whose cell boundaries along the sweep are ``x_cb`` (Ns + 1
    increasing values, ghost cells included), as Fortran-ordered host arrays
    of the harness layouts (NC = Ns - 6).  Computed by the library
    (weno_sb_coefficients): MFC's s_compute_weno_coefficients, which the
    reference replaces by synthetic values (f90:246-279)."""
    x = np.ascontiguousarray(x_cb, dtype=np.float64)
    ns = x.size - 1
    nc = ns - 6
    if nc < 1:
        raise ValueError(f"need at least 7 cells (got {ns})")
    pL = np.zeros((nc, 5, 3), order="F")
    pR = np.zeros((nc, 5, 3), order="F")
    dL = np.zeros((5, nc), order="F")
    dR = np.zeros((5, nc), order="F")
    bc = np.zeros((nc, 5, 6), order="F")
    L.check(L.lib().weno_sb_coefficients(int(order), ns, x.ctypes.data, pL.ctypes.data, pR.ctypes.data,
                                         dL.ctypes.data, dR.ctypes.data, bc.ctypes.data))
    return pL, pR, dL, dR, bc


def stretched_boundaries(cells: int, buff: int, ratio: float = 4.0, centre: float = 0.5, width: float = 0.1):
    """Cell boundaries of one axis with `cells` interior cells on [0, 1] and
    `buff` ghost cells per side (mirrored widths): a tanh refinement centred
    on `centre`, whose cells are up to `ratio` times narrower there than
    far away (the kind of grid MFC clusters around a feature).  Returns
    cells + 2 buff + 1 increasing values (the sweep's Ns + 1 boundaries)."""
    s = np.linspace(0.0, 1.0, 4097)
    dens = 1.0 + (ratio - 1.0) * (1.0 - np.tanh((s - centre) / width) ** 2)
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * np.diff(s))])
    cum /= cum[-1]
    inner = np.interp(np.linspace(0.0, 1.0, cells + 1), cum, s)
    w = np.diff(inner)
    left = inner[0] - np.cumsum(w[:buff])[::-1]
    right = inner[-1] + np.cumsum(w[::-1][:buff])
    return np.concatenate([left, inner, right])
