"""Pin of the oracle's per-mode spectral maps against the reference's own
code: the reference's CUDA twins linearized_kernel / linearizedIteratekernel
(CUDA_WRAP/linearized.cu, compiled from the reference sources into
oracle/_ref/ by oracle/Makefile) run on random spectra and are compared with
the oracle's predictor / corrector restatement
(movefieldshydrolinlayersplit.cpp:808-900, :1374-1477).  The reference is
compiled with FMA contraction and the oracle without, so agreement is to a
few FP64 ulp."""
import ctypes as C

import numpy as np
import pytest

from oracle import binding

pytestmark = pytest.mark.gpu

TOL = 1e-13


def ref_or_skip():
    L = binding.reference_lib()
    if L is None:
        pytest.skip("reference twins not built (no reference checkout where build() ran)")
    return L


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def ptrs(ts):
    return (C.c_void_p * len(ts))(*[C.c_void_p(t.data_ptr()) for t in ts])


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("n", [32, 64])
def test_predictor_matches_reference_twin(n):
    import torch
    L = ref_or_skip()
    rng = np.random.default_rng(n)
    N = n * n
    hx, dens, ylen, zlen = 0.05, 1.0, n * 0.05, n * 0.05
    P = {k: rng.standard_normal(N) for k in ("RhoP", "JxP", "JyP", "JzP", "ExP", "EyP", "EzP")}
    beam = {k: rng.standard_normal(N) for k in ("RhoBeam", "RhoBeamP", "JxBeam", "JxBeamP")}
    want = binding.predictor_modes(n, n, hx, dens, ylen, zlen, P, beam)
    # CUDA_WRAP_linearized_loop reads the P spectra from the C arrays
    # (Rho, Jx, Jy, Jz, Ex, Ey, Ez) and copies them into the P arrays
    z = np.zeros(N)
    t = [dev(torch, P["RhoP"]), dev(torch, z), dev(torch, z), dev(torch, z), dev(torch, z),
         dev(torch, P["ExP"]), dev(torch, P["EyP"]), dev(torch, P["EzP"]), dev(torch, z),
         dev(torch, z), dev(torch, z), dev(torch, P["JxP"]), dev(torch, P["JyP"]),
         dev(torch, P["JzP"]), dev(torch, z), dev(torch, z), dev(torch, z),
         dev(torch, beam["JxBeam"]), dev(torch, beam["RhoBeam"]), dev(torch, beam["JxBeamP"]),
         dev(torch, beam["RhoBeamP"])]
    assert L.ref_linearized_loop(n, n, hx, dens, zlen, ylen, ptrs(t)) == 0
    got = {"Rho": t[0], "Ex": t[5], "Ey": t[6], "Ez": t[7], "Jx": t[11], "Jy": t[12],
           "Jz": t[13], "Bx": t[14], "By": t[15], "Bz": t[16]}
    for k, v in got.items():
        assert rel(v.cpu().numpy(), want[k]) < TOL, k


@pytest.mark.parametrize("n", [32, 64])
def test_corrector_matches_reference_twin(n):
    import torch
    L = ref_or_skip()
    rng = np.random.default_rng(100 + n)
    N = n * n
    hx, dens, ylen, zlen = 0.05, 1.0, n * 0.05, n * 0.05
    P = {k: rng.standard_normal(N) for k in ("RhoP", "JxP", "JyP", "JzP", "EyP", "EzP")}
    beam = {k: rng.standard_normal(N) for k in ("RhoBeam", "RhoBeamP", "JxBeam", "JxBeamP")}
    J = {k: rng.standard_normal(N) for k in ("Jx", "Jy", "Jz")}
    rho_old = rng.standard_normal(N)
    want = binding.corrector_modes(n, n, hx, dens, ylen, zlen, P, beam, J, rho_old)
    z = np.zeros(N)
    t = [dev(torch, rho_old), dev(torch, P["RhoP"]), dev(torch, P["JxP"]), dev(torch, P["JyP"]),
         dev(torch, P["JzP"]), dev(torch, z), dev(torch, z), dev(torch, z), dev(torch, P["EyP"]),
         dev(torch, P["EzP"]), dev(torch, J["Jx"]), dev(torch, J["Jy"]), dev(torch, J["Jz"]),
         dev(torch, z), dev(torch, z), dev(torch, z), dev(torch, beam["JxBeam"]),
         dev(torch, beam["RhoBeam"]), dev(torch, beam["JxBeamP"]), dev(torch, beam["RhoBeamP"])]
    assert L.ref_linearized_iterate_loop(n, n, hx, dens, zlen, ylen, ptrs(t)) == 0
    got = {"Rho": t[0], "Ex": t[5], "Ey": t[6], "Ez": t[7], "Bx": t[13], "By": t[14],
           "Bz": t[15]}
    for k, v in got.items():
        assert rel(v.cpu().numpy(), want[k]) < TOL, k
