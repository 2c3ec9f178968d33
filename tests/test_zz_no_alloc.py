"""sqb200_jk_build_noalloc: the J/K build for callers that cannot allocate GPU memory (their
device memory belongs to their own allocator, or they cannot afford cudaMalloc's implicit
synchronisation).  Its scratch lives in a static device array, so it must give the same J and
K as the regular entry point -- also on a second call, which finds the first call's leftovers
in that array -- and its first call must also match the reference's own build stored in the
fixture.  This file is collected last on purpose."""
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


def _noalloc(L, eng, PA, PB, restricted, outs, stream, cutoff=1e-10):
    JT, KA, KB = outs
    for o in outs:
        if o is not None:
            o.fill_(float("nan"))                  # every element must be written
    return L.sqb200_jk_build_noalloc(eng._ctx, PA.data_ptr(), PB.data_ptr(), int(restricted), cutoff, cutoff,
                                     float("inf"), JT.data_ptr(), KA.data_ptr(),
                                     None if KB is None else KB.data_ptr(), stream)


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
    for call, (PAh, PBh) in enumerate(dens):
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
        if call == 0:
            # the fixture's density: the reference's own direct-mode build (density screen on
            # every quartet, as dscreen_rmax = inf asks)
            assert np.abs(JT - g["JT_dir"]).max() <= TOL
            assert np.abs(KA - g["KA_dir"]).max() <= TOL
            assert np.abs(KB - g["KB_dir"]).max() <= TOL
    eng.close()


@pytest.mark.gpu
def test_noalloc_takes_no_device_memory_and_accepts_null_kb():
    """Free device memory is unchanged across a call (made after a first call, which may load
    kernel code under lazy module loading), and a restricted call may pass KB = NULL."""
    import torch
    sqb, L = _lib()
    g = golden("h2co_631gs")
    eng = sqb.JKEngine(golden_basis(g), schwarz=g["schwarz"])
    dev = torch.device("cuda:0")
    n = eng.nbf
    PA = torch.tensor(g["PA"], dtype=torch.float64, device=dev)
    outs = (torch.empty((n, n), dtype=torch.float64, device=dev),
            torch.empty((n, n), dtype=torch.float64, device=dev), None)
    assert _noalloc(L, eng, PA, PA, True, outs, None) == 0, L.sqb200_last_error().decode()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    assert _noalloc(L, eng, PA, PA, True, outs, None) == 0, L.sqb200_last_error().decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    JT, KA = outs[0].cpu().numpy(), outs[1].cpu().numpy()
    assert np.abs(JT - g["JT_dir"]).max() <= TOL and np.abs(KA - g["KA_dir"]).max() <= TOL
    eng.close()


@pytest.mark.gpu
def test_noalloc_rejects_inputs_beyond_its_limit():
    import torch
    sqb, L = _lib()
    dev = torch.device("cuda:0")
    # 540 functions > 256
    atoms = sqb.molecules.to_bohr(sqb.molecules.c60())
    b = sqb.basis.build_basis(atoms, "631g")
    eng = sqb.JKEngine(b, schwarz=np.ones((b.nbf, b.nbf)))
    n = b.nbf
    PA = torch.zeros((n, n), dtype=torch.float64, device=dev)
    outs = tuple(torch.empty((n, n), dtype=torch.float64, device=dev) for _ in range(3))
    rc = _noalloc(L, eng, PA, PA, True, outs, None)
    assert rc == -1
    assert b"exceed its limit of 256" in L.sqb200_last_error()
    eng.close()
    # 250 functions, but with no Schwarz cutoff every pair of shell pairs is a quartet: far more
    # than 65,536 work items
    atoms = sqb.molecules.to_bohr(sqb.molecules.random_organic(np.random.default_rng(1), 14))
    b = sqb.basis.build_basis(atoms, "6-31g*")
    assert b.nbf <= 256
    eng = sqb.JKEngine(b)
    n = b.nbf
    PA = torch.zeros((n, n), dtype=torch.float64, device=dev)
    outs = tuple(torch.empty((n, n), dtype=torch.float64, device=dev) for _ in range(3))
    rc = _noalloc(L, eng, PA, PA, True, outs, None, cutoff=0.0)
    assert rc == -1
    assert b"work items exceed its limit of 65536" in L.sqb200_last_error()
    eng.close()
