"""The restart loader (-sfile): the reference's LoadData mapping by default, and the
opt-in faithful mapping (-restart-faithful) that reloads the last written level into
the state it came from.  Host only."""
import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import __main__ as cli
from multiblockmomentsfv_b200 import blockfile as bf
from multiblockmomentsfv_b200 import output


def _levels(d, seed):
    rng = np.random.default_rng(seed)
    return [[H.random_layer(rng, b) for b in d.blocks] for _ in range(2)]


def _ring(U, b):
    return U[2:b.ny + 4, 2:b.nx + 4]


def test_faithful_restart_reloads_the_last_level(tmp_path):
    d = H.deck("squareSmall")
    lv = _levels(d, 1)
    w = output.Writer(str(tmp_path), d, "Riemann2D", single=False)
    w.write(lv[0], 0.0, -1)
    w.write(lv[1], 0.1, 5)
    got = cli.load_restart(d, w.base, faithful=True)
    for b, blk in enumerate(d.blocks):
        a, ref = _ring(got[b], blk), _ring(lv[1][b], blk)
        assert np.allclose(a, ref, rtol=1e-12, atol=1e-14), np.abs(a - ref).max()
        # outside the interior plus one ghost ring the layer stays zero (set by the ghost fill)
        assert not got[b][0].any() and not got[b][:, 0].any()


def test_default_restart_keeps_the_references_mapping(tmp_path):
    """The reference's LoadData puts the stored p where theta belongs and P_ij where
    T_ij belongs, and reads the first level: a state at rest with rho = 2, theta = 1
    comes back with theta = p = 2 and T_ii = P_ii = 2."""
    d = H.deck("squareSmall")
    lv = []
    for b in d.blocks:
        U = np.zeros((b.nyp, b.nxp, bf.NV))
        U[..., 0] = 2.0
        U[..., 3] = 1.5 * 2.0          # E = 3/2 rho theta
        U[..., 4] = 2.0                # rho T11
        U[..., 6] = 2.0
        lv.append(U)
    w = output.Writer(str(tmp_path), d, "Riemann2D", single=False)
    w.write(lv, 0.0, -1)
    w.write([U * 1.1 for U in lv], 0.1, 5)
    got = cli.load_restart(d, w.base)
    for b, blk in enumerate(d.blocks):
        a = _ring(got[b], blk)
        assert np.allclose(a[..., 0], 2.0)
        assert np.allclose(a[..., 3], 1.5 * 2.0 * 2.0)      # theta taken as p = 2
        assert np.allclose(a[..., 4], 2.0 * 2.0)            # T11 taken as P11 = 2


def _reference_load(d, path):
    """The reference's own LoadData (src/Mesh.c:198-283, oracle/_ref/libmbmref.so)
    into DB_Block layers whose L_DATA starts at zero, as main allocates it."""
    import ctypes as C
    import os
    import sys
    import pytest
    sys.path.insert(0, os.path.join(H.HERE, "..", "oracle"))
    import oracle as O
    if O.ref_lib() is None:
        pytest.skip("reference sources not built here")
    ref = O.Reference(d)
    O.ref_lib().LoadData.argtypes = [C.POINTER(O.DBBlock), C.c_int, C.c_char_p]
    O.ref_lib().LoadData(ref.B, len(d.blocks), path.encode())
    return [ref.get_layer(O.DATA, b) for b in range(len(d.blocks))]


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("deck", ["squareSmall", "Lshape"])
def test_default_restart_equals_reference_loaddata(tmp_path, deck, single):
    """The package's restart loader (default mapping) against the reference's own
    LoadData on the same file: every cell of L_DATA bit for bit, on a two-level
    result file (the first level is read) in both payload precisions."""
    d = H.deck(deck)
    lv = _levels(d, 3 + single)
    w = output.Writer(str(tmp_path), d, "Riemann2D", single=single)
    w.write(lv[0], 0.0, -1)
    w.write(lv[1], 0.1, 5)
    for name in (w.base, w.hdr, w.dat):        # basename, .hdr or .dat, as LoadData accepts
        ref = _reference_load(d, name)
        got = cli.load_restart(d, name)
        for b in range(len(d.blocks)):
            H.assert_bitwise(got[b], ref[b], f"{deck} block {b + 1} ({name[-4:]})")


@pytest.mark.parametrize("single", [False, True])
def test_restart_payloads_as_stored(tmp_path, single):
    """The zones the device loader receives (cli.restart_payloads): the file's values in
    the file's precision, the first level by default and the last with faithful."""
    d = H.deck("squareSmall")
    lv = _levels(d, 9 + single)
    w = output.Writer(str(tmp_path), d, "Riemann2D", single=single)
    w.write(lv[0], 0.0, -1)
    w.write(lv[1], 0.1, 5)
    zones, _ = output.read(w.base)
    nb = len(d.blocks)
    for faithful, sel in ((False, zones[:nb]), (True, zones[nb:])):
        got = cli.restart_payloads(d, w.base, faithful=faithful)
        for b, (p, z) in enumerate(zip(got, sel)):
            assert p.dtype == (np.float32 if single else np.float64)
            assert p.shape == ((d.blocks[b].nx + 2) * (d.blocks[b].ny + 2), 10)
            H.assert_bitwise(p.astype(np.float64), z["values"], f"block {b + 1}")
