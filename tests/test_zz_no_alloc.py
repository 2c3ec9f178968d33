"""sqb200_jk_build_noalloc: the J/K build for callers that cannot allocate GPU memory (their
device memory belongs to their own allocator, or they cannot afford cudaMalloc's implicit
synchronisation).  Its scratch lives in a static device array, so it must give the same J and
K as the regular entry point -- also on a second call, which finds the first call's leftovers
in that array.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from conftest import golden, golden_basis, load_sqb200

TOL = 1e-10


def _lib():
    sqb = load_sqb200()
    L = sqb.load_library()
    vp = ctypes.c_void_p
    L.sqb200_jk_build_noalloc.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, vp, vp, vp, vp]
    L.sqb200_jk_build_noalloc.restype = ctypes.c_int
    return sqb, L


def _noalloc(L, eng, PA, PB, restricted, outs, stream):
    JT, KA, KB = outs
    for o in outs:
        o.fill_(float("nan"))                      # every element must be written
    return L.sqb200_jk_build_noalloc(eng._ctx, PA.data_ptr(), PB.data_ptr(), int(restricted), 1e-10, 1e-10,
                                     float("inf"), JT.data_ptr(), KA.data_ptr(), KB.data_ptr(), stream)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["benzene_631gs", "oh_321g_uhf"])
def test_noalloc_matches_regular_entry_point_twice(case):
    import torch
    sqb, L = _lib()
    g = golden(case)
    restricted = bool(g["restricted"])
    eng = sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    dev = torch.device("cuda:0")
    st = torch.cuda.Stream(dev)
    rng = np.random.default_rng(1)
    n = eng.nbf
    # two different densities on two calls in a row
    dens = [(g["PA"], g["PB"])]
    E = rng.normal(size=(n, n)) * 1e-3
    dens.append((g["PA"] + E + E.T, g["PB"] - E - E.T))
    outs = tuple(torch.empty((n, n), dtype=torch.float64, device=dev) for _ in range(3))
    for PAh, PBh in dens:
        JT0, KA0, KB0 = eng.build(PAh, None if restricted else PBh, restricted=restricted, scf_cutoff=1e-10)
        PA = torch.tensor(PAh, dtype=torch.float64, device=dev)
        PB = PA if restricted else torch.tensor(PBh, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = _noalloc(L, eng, PA, PB, restricted, outs, st.cuda_stream)
        assert rc == 0, L.sqb200_last_error().decode()
        st.synchronize()
        JT, KA, KB = (o.cpu().numpy() for o in outs)
        assert np.abs(JT - JT0).max() <= TOL
        assert np.abs(KA - KA0).max() <= TOL
        assert np.abs(KB - KB0).max() <= TOL
    eng.close()


@pytest.mark.gpu
def test_noalloc_rejects_inputs_beyond_its_limit():
    import torch
    sqb, L = _lib()
    atoms = sqb.molecules.to_bohr(sqb.molecules.c60())
    b = sqb.basis.build_basis(atoms, "631g")            # 540 functions > 256
    eng = sqb.JKEngine(b, schwarz=np.ones((b.nbf, b.nbf)))
    dev = torch.device("cuda:0")
    n = b.nbf
    PA = torch.zeros((n, n), dtype=torch.float64, device=dev)
    outs = tuple(torch.empty((n, n), dtype=torch.float64, device=dev) for _ in range(3))
    rc = _noalloc(L, eng, PA, PA, True, outs, None)
    assert rc == -1
    assert b"exceed its limit of 256" in L.sqb200_last_error()
    eng.close()
