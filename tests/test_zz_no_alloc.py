"""mbm_stage_noalloc -- one Heun stage on device buffers the caller owns, with the
kernel's scratch in a fixed device array -- against the allocating context path
(mbm_update), through the C ABI.  Callers of it cannot allocate device memory (a
memory pool owns the GPU, or every allocation is fixed at start-up); here the test
plays that caller and owns the buffers (torch tensors).

Two different stage calls in a row, then the first again: the shared scratch
keeps the previous call's contents, so a call that failed to clear it would show.
The comparison is bit for bit, the tolerance every parity test here uses."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import _abi, scenario as sc, solver as sv

pytestmark = pytest.mark.gpu


def plane_layout(blocks):
    """The library's device layout (include/mbm_b200.h, mbm_stage_noalloc)."""
    offs, total = [], 0
    for b in blocks:
        nxp, nyp = b.nx + 6, b.ny + 6
        pitch = (nxp + 1 + 3) // 4 * 4
        plane = (pitch * nyp + 31) // 32 * 32
        offs.append((total, pitch, plane))
        total += 9 * plane
    return offs, total


def to_planes(layers, offs, total):
    buf = np.zeros(total)
    for U, (off, pitch, plane) in zip(layers, offs):
        nyp, nxp = U.shape[:2]
        for m in range(9):
            buf[off + m * plane: off + m * plane + nyp * pitch].reshape(nyp, pitch)[:, 1:nxp + 1] = U[:, :, m]
    return buf


def from_planes(buf, blocks, offs):
    out = []
    for b, (off, pitch, plane) in zip(blocks, offs):
        nxp, nyp = b.nx + 6, b.ny + 6
        U = np.empty((nyp, nxp, 9))
        for m in range(9):
            U[:, :, m] = buf[off + m * plane: off + m * plane + nyp * pitch].reshape(nyp, pitch)[:, 1:nxp + 1]
        out.append(U)
    return out


def test_stage_noalloc_matches_context_path():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    rng = np.random.default_rng(42)
    d = H.quadrant_deck(40, Kn=0.01, limiter=4)
    data = [H.random_layer(rng, b) for b in d.blocks]
    tmp = [H.random_layer(rng, b) for b in d.blocks]
    dt = 0.003

    # the existing entry points: mbm_update on a context
    with sv.Solver(d, sc.Scenario.seeded_quadrant(1)) as s:
        for b in range(len(d.blocks)):
            s.upload(sv.L_DATA, b, data[b])
            s.upload(sv.L_TMP, b, tmp[b])
        cfl1 = s.update(sv.L_TMP, sv.L_DATA, sv.L_DATA, dt, 0.0, 0)
        ref1 = [H.interior(s.download(sv.L_TMP, b)) for b in range(len(d.blocks))]
        for b in range(len(d.blocks)):
            s.upload(sv.L_TMP, b, tmp[b])
        cfl2 = s.update(sv.L_NEW, sv.L_TMP, sv.L_DATA, dt, 0.0, 1)
        ref2 = [H.interior(s.download(sv.L_NEW, b)) for b in range(len(d.blocks))]

    L = _abi.lib()
    descs = _abi.block_descs(d.blocks)
    offs, total = plane_layout(d.blocks)
    d_data = torch.from_numpy(to_planes(data, offs, total)).cuda()
    d_tmp = torch.from_numpy(to_planes(tmp, offs, total)).cuda()
    stream = torch.cuda.current_stream().cuda_stream

    def call(inp, data0, heun):
        out = torch.zeros(total, dtype=torch.float64, device="cuda")
        cfl = np.zeros(len(d.blocks))
        st = L.mbm_stage_noalloc(descs, len(d.blocks), inp.data_ptr(), data0.data_ptr() if data0 is not None else None,
                                 out.data_ptr(), d.Kn, d.F, d.limiter, dt, heun,
                                 cfl.ctypes.data_as(C.POINTER(C.c_double)), stream)
        assert st == _abi.MBM_OK, L.mbm_last_error(None).decode()
        return [H.interior(U) for U in from_planes(out.cpu().numpy(), d.blocks, offs)], cfl

    for _ in range(2):     # both stages, twice, on the shared scratch
        got1, c1 = call(d_data, None, 0)
        got2, c2 = call(d_tmp, d_data, 1)
        H.assert_bitwise(c1, cfl1, "stage-1 CFL")
        H.assert_bitwise(c2, cfl2, "stage-2 CFL")
        for b in range(len(d.blocks)):
            H.assert_bitwise(got1[b], ref1[b], f"stage 1 block {b}")
            H.assert_bitwise(got2[b], ref2[b], f"stage 2 block {b}")


def test_stage_noalloc_rejects_oversize():
    """Blocks beyond the scratch limit are refused before anything touches the GPU."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    L = _abi.lib()
    from multiblockmomentsfv_b200 import blockfile as bf
    big = [bf.Block(1, 0.0, 1.0, 0.0, 1.0, 8192, 8192, (0, 0, 0, 0))]
    tiny = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = L.mbm_stage_noalloc(_abi.block_descs(big), 1, tiny.data_ptr(), None, tiny.data_ptr(), 0.01, 0.0, 4,
                             1e-4, 0, None, None)
    assert st == _abi.MBM_EINVAL
    assert b"scratch limit" in L.mbm_last_error(None)


def test_stage_noalloc_reports_nonfinite():
    """A NaN in one input cell makes the stage write NaNs; the call says so with
    MBM_ENONFINITE (a NaN never enters the CFL maxima, so the CFL values alone would
    not show it), and the next call on a finite input is MBM_OK again, because each
    call clears the flag in the shared scratch."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    rng = np.random.default_rng(7)
    d = H.quadrant_deck(24, Kn=0.01, limiter=4)
    data = [H.random_layer(rng, b) for b in d.blocks]
    L = _abi.lib()
    descs = _abi.block_descs(d.blocks)
    offs, total = plane_layout(d.blocks)
    stream = torch.cuda.current_stream().cuda_stream
    good = torch.from_numpy(to_planes(data, offs, total)).cuda()
    data[1][10, 12, 3] = float("nan")
    bad = torch.from_numpy(to_planes(data, offs, total)).cuda()
    out = torch.zeros(total, dtype=torch.float64, device="cuda")
    cfl = np.zeros(len(d.blocks))
    for inp, want in ((bad, _abi.MBM_ENONFINITE), (good, _abi.MBM_OK), (bad, _abi.MBM_ENONFINITE)):
        st = L.mbm_stage_noalloc(descs, len(d.blocks), inp.data_ptr(), None, out.data_ptr(), d.Kn, d.F,
                                 d.limiter, 1e-3, 0, cfl.ctypes.data_as(C.POINTER(C.c_double)), stream)
        assert st == want, (st, L.mbm_last_error(None))
        assert np.isfinite(cfl).all()
