"""The allocation-free step entry point (tlm_step_planes_noalloc).

It exists for callers that may not allocate device memory themselves (a host
that owns the GPU's memory in its own pool, or a time-critical loop that must
not pay cudaMalloc's device-wide synchronisation). They own the pulse planes
and the library advances them with scratch kept in a fixed static device
array. This test drives it through the C ABI on buffers the test allocates
(as such a caller would) and checks two calls in a row against the regular
handle-based entry point on the same state: pulse state and stubs bitwise,
energy within the energy tolerance the other GPU tests use (relative 1e-6),
in the regular and in the bounds-checked build of the library, and checks
that further calls leave the device's free memory unchanged.
"""
import ctypes as C

import numpy as np
import pytest

from emsolver_b200 import MatProps, TlmConfig, TlmSolver, VoxelGridSpec, _lib

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-6
PADX = 8


def grid_case():
    """13x9x11 (x extent not a multiple of the vector width), two lossy
    dielectric boxes, 6 % PEC, outer reflection 0.5."""
    nx, ny, nz = 13, 9, 11
    rng = np.random.default_rng(21)
    mat = np.zeros((nz, ny, nx), np.uint8)
    mat[2:7, 1:6, 3:10] = 2
    mat[5:10, 4:9, 0:5] = 3
    mat[rng.random((nz, ny, nx)) < 0.06] = 1
    table = [MatProps(4.5, 0.02), MatProps(2.0, 0.0)]
    v0 = rng.standard_normal(nx * ny * nz * 12).astype(np.float32)
    v0.reshape(-1, 12)[mat.reshape(-1) == 1] = 0.0
    return nx, ny, nz, mat, table, np.float32(0.5), v0


def to_planes(aos, nx, ny, nz):
    """AoS (cell*12 + slot) -> 12 padded planes, padding zero."""
    px = -(-nx // PADX) * PADX
    pl = np.zeros((12, nz, ny, px), np.float32)
    pl[:, :, :, :nx] = aos.reshape(nz, ny, nx, 12).transpose(3, 0, 1, 2)
    return pl


def connect(refl, mat_p, nx, ny, nz, rho):
    """Incident pulses from reflected planes: the reference's connect
    (TlmSolver.cpp:551-613) as a gather, in float32; returns AoS."""
    refl = refl[:, :, :, :nx]
    pec = mat_p[:, :, :nx] == 1
    inc = np.zeros_like(refl)
    for s in range(12):
        a, side = s >> 2, (s >> 1) & 1
        own = refl[s]
        src = refl[s ^ 2]
        out = np.empty_like(own)
        sl_all = [slice(None)] * 3
        axis = 2 - a                     # planes are [k][j][i]
        n = (nz, ny, nx)[axis]
        # neighbour value and neighbour PEC flag, shifted along the axis
        nb = np.zeros_like(own)
        nbpec = np.zeros_like(pec)
        lo, hi = list(sl_all), list(sl_all)
        if side == 1:
            lo[axis], hi[axis] = slice(0, n - 1), slice(1, n)
        else:
            lo[axis], hi[axis] = slice(1, n), slice(0, n - 1)
        nb[tuple(lo)] = src[tuple(hi)]
        nbpec[tuple(lo)] = pec[tuple(hi)]
        outside = np.zeros_like(pec)
        edge = list(sl_all)
        edge[axis] = n - 1 if side == 1 else 0
        outside[tuple(edge)] = True
        out[...] = nb
        out[nbpec] = -own[nbpec]
        out[outside] = rho * own[outside]
        out[pec] = 0.0
        inc[s] = out
    return inc.transpose(1, 2, 3, 0).reshape(-1)


@pytest.mark.parametrize("variant", ["", "checked"])
def test_no_alloc_step_matches_handle_step(built, variant):
    torch = pytest.importorskip("torch")
    nx, ny, nz, mat, table, rho, v0 = grid_case()
    g = VoxelGridSpec(nx, ny, nz)

    # the regular entry point: handle, library-owned memory
    s = TlmSolver()
    s.setup(g, mat.reshape(-1), table, TlmConfig(boundaryRho=float(rho), totalSteps=2))
    s.setPulses(v0)
    s.step(1)
    inc1 = s.pulses()
    _, e_hist = s.getEnergyHistory(f64=True)
    s.step(1)
    inc2 = s.pulses()
    stubs2 = s.stubs()
    yhat, ghat = s.tables()
    s.close()

    # the allocation-free entry point on buffers the caller owns
    px = -(-nx // PADX) * PADX
    P = px * ny * nz
    dev = torch.device("cuda", 0)
    a = torch.from_numpy(to_planes(v0, nx, ny, nz).reshape(-1)).to(dev)
    b = torch.zeros(12 * P, dtype=torch.float32, device=dev)
    stub = torch.zeros(3 * P, dtype=torch.float32, device=dev)
    mat_p = np.ones((nz, ny, px), np.uint8)
    mat_p[:, :, :nx] = mat
    dmat = torch.from_numpy(mat_p.reshape(-1)).to(dev)
    dy = torch.from_numpy(yhat).to(dev)
    dg = torch.from_numpy(ghat).to(dev)
    energy = torch.zeros(2, dtype=torch.float64, device=dev)
    L = _lib.load(variant)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def call(src, dst, incident, eslot):
        st = L.tlm_step_planes_noalloc(src.data_ptr(), dst.data_ptr(), stub.data_ptr(),
                                       dmat.data_ptr(), dy.data_ptr(), dg.data_ptr(), len(table),
                                       nx, ny, nz, float(rho), incident,
                                       energy.data_ptr() + 8 * eslot, stream)
        assert st == _lib.TLM_OK, L.tlm_last_error(None)

    call(a, b, 1, 0)        # step 0: incident state in, reflected out
    call(b, a, 0, 1)        # step 1: reflected in, reflected out
    torch.cuda.synchronize(dev)
    refl0 = b.cpu().numpy().reshape(12, nz, ny, px)
    refl1 = a.cpu().numpy().reshape(12, nz, ny, px)
    e = energy.cpu().numpy()


    assert np.array_equal(connect(refl0, mat_p, nx, ny, nz, rho), inc1)
    assert np.array_equal(connect(refl1, mat_p, nx, ny, nz, rho), inc2)
    st = stub.cpu().numpy().reshape(3, nz, ny, px)[:, :, :, :nx].transpose(1, 2, 3, 0).reshape(-1)
    assert np.array_equal(st, stubs2)
    assert abs(e[0] - e_hist[0]) <= ENERGY_RTOL * e_hist[0]
    ref1 = float(np.sum(inc1.astype(np.float64) ** 2))
    assert abs(e[1] - ref1) <= ENERGY_RTOL * ref1

    # further calls (every kernel already loaded by the two above) leave the
    # device's free memory where it was: the entry point allocates nothing
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    for r in range(4):
        call(a if r % 2 == 0 else b, b if r % 2 == 0 else a, r & 1, 0)
    torch.cuda.synchronize(dev)
    assert torch.cuda.mem_get_info(dev)[0] == free0


def test_no_alloc_rejects_oversized_grid(built):
    """Sizes beyond the static scratch are refused before anything runs."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(64, dtype=torch.float32, device=dev)
    out = torch.zeros(64, dtype=torch.float32, device=dev)
    m = torch.zeros(64, dtype=torch.uint8, device=dev)
    L = _lib.load()
    st = L.tlm_step_planes_noalloc(buf.data_ptr(), out.data_ptr(), None, m.data_ptr(), None, None, 0,
                                   1024, 1024, 128, 0.0, 0, None, None)
    assert st == _lib.TLM_EINVAL
    assert b"at most 67108864" in L.tlm_last_error(None)
    # extents whose product would overflow 64 bits are refused the same way
    st = L.tlm_step_planes_noalloc(buf.data_ptr(), out.data_ptr(), None, m.data_ptr(), None, None, 0,
                                   2**31 - 1, 2**31 - 1, 2**31 - 1, 0.0, 0, None, None)
    assert st == _lib.TLM_EINVAL


def test_no_alloc_rejects_missing_tables(built):
    """A dielectric table without its stubs or entries is refused before
    anything runs (the step would otherwise read through a null pointer)."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(12 * 8 * 8 * 8, dtype=torch.float32, device=dev)
    out = torch.zeros_like(buf)
    stub = torch.zeros(3 * 8 * 8 * 8, dtype=torch.float32, device=dev)
    tab = torch.ones(4, dtype=torch.float32, device=dev)
    m = torch.zeros(8 * 8 * 8, dtype=torch.uint8, device=dev)
    L = _lib.load()
    def ptr(t):
        return None if t is None else t.data_ptr()

    for stubs, yh, gh in ((stub, None, tab), (stub, tab, None), (None, tab, tab)):
        st = L.tlm_step_planes_noalloc(buf.data_ptr(), out.data_ptr(), ptr(stubs), m.data_ptr(),
                                       ptr(yh), ptr(gh), 1, 8, 8, 8, 0.0, 0, None, None)
        assert st == _lib.TLM_EINVAL
    st = L.tlm_step_planes_noalloc(buf.data_ptr(), out.data_ptr(), None, m.data_ptr(), None, None, -1,
                                   8, 8, 8, 0.0, 0, None, None)
    assert st == _lib.TLM_EINVAL


def test_no_alloc_ids_past_the_table_step_to_nan(built):
    """Material ids past the caller's table make those nodes' pulses NaN
    (the padded static table), while every other node steps as usual."""
    torch = pytest.importorskip("torch")
    nx, ny, nz = 8, 8, 8
    P = nx * ny * nz
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    mat = np.zeros((nz, ny, nx), np.uint8)
    mat[4, 4, 4] = 3                       # id 3: past a one-entry table
    mat[1, 1, 1] = 2
    v0 = rng.standard_normal(12 * P).astype(np.float32)
    a = torch.from_numpy(v0).to(dev)
    b = torch.zeros_like(a)
    stub = torch.zeros(3 * P, dtype=torch.float32, device=dev)
    tab = torch.tensor([4.0], dtype=torch.float32, device=dev)
    dmat = torch.from_numpy(mat.reshape(-1)).to(dev)
    L = _lib.load()
    st = L.tlm_step_planes_noalloc(a.data_ptr(), b.data_ptr(), stub.data_ptr(), dmat.data_ptr(),
                                   tab.data_ptr(), tab.data_ptr(), 1, nx, ny, nz, 0.0, 1, None, None)
    assert st == _lib.TLM_OK, L.tlm_last_error(None)
    torch.cuda.synchronize(dev)
    out = b.cpu().numpy().reshape(12, P)
    bad = (4 * ny + 4) * nx + 4
    assert np.all(np.isnan(out[:, bad]))
    assert np.all(np.isfinite(np.delete(out, bad, axis=1)))
