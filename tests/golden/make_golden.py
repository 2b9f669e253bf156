"""Generate the transform golden vectors in tests/golden/dtt_golden.npz.

The reference runs FFTW's REDFT11 / RODFT11 (movefieldshydrolinlayersplit.cpp
:389-427); scipy.fft's dct/dst type 4 implement the same published
definitions (FFTW manual, "1d Real-even DFTs (DCTs)" / "1d Real-odd DFTs
(DSTs)"), unnormalised: Y_k = 2 sum_j X_j cos|sin(pi (j+1/2)(k+1/2)/n).
Inputs: seeded normals, and the reference's own harness pattern of
surfaceFFT.cu:402-412 (x[i][j] = 10 i + j and -10 i + j).
Run:  python tests/golden/make_golden.py
"""
import os

import numpy as np
import scipy.fft as sf

HERE = os.path.dirname(os.path.abspath(__file__))


def t2(x, kz, ky):
    fy = sf.dct if ky == 0 else sf.dst
    fz = sf.dct if kz == 0 else sf.dst
    return fz(fy(x, type=4, axis=1), type=4, axis=0)


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    for n in (1, 2, 3, 5, 8, 16, 24, 64, 128):
        x = rng.standard_normal(n)
        out[f"d1_in_{n}"] = x
        out[f"d1_dct4_{n}"] = sf.dct(x, type=4)
        out[f"d1_dst4_{n}"] = sf.dst(x, type=4)
    for (nz, ny) in ((4, 4), (8, 16), (32, 32), (16, 48)):
        x = rng.standard_normal((nz, ny))
        out[f"d2_in_{nz}x{ny}"] = x
        for kz in (0, 1):
            for ky in (0, 1):
                out[f"d2_{kz}{ky}_{nz}x{ny}"] = t2(x, kz, ky)
    # the reference harness inputs (4 x 4 and 8 x 8)
    for n in (4, 8):
        i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        # plan2D: (RODFT11, REDFT11) on 10 i + j; plan2D_1: (REDFT11, RODFT11)
        # on -10 i + j (surfaceFFT.cu:402-403)
        for sign, tag, kz, ky in ((1, "p", 1, 0), (-1, "m", 0, 1)):
            x = (sign * 10.0 * i + j).astype(np.float64)
            out[f"harness_{tag}_{n}_in"] = x
            out[f"harness_{tag}_{n}_out"] = t2(x, kz, ky)
    np.savez_compressed(os.path.join(HERE, "dtt_golden.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
