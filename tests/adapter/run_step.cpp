// A driver of the MeshQS adapter (include/mesh_qs.h) as the reference's
// Domain::Step would use it: read a deck and its inputs from a binary file,
// load the beam and the front plasma, run `steps` beam steps
// (MoveBeamParticles + MoveAllSplitLayers), write the on-axis Ex of every
// layer.
//
//   run_step <inputs.bin> <onaxis_out.bin>
//
// inputs.bin: int32 My, Mz, Mx, nIter, NxSplit, ppc, precision, shape, steps;
// float64 Hx, Hy, Hz, Ts, density, wavelength; int64 nb, then the beam (int32
// i, j, k [nb], float64 x, y, z, px, py, pz, w [nb]); int64 np, then the
// front plasma (int32 cell [np], float64 y, z, px, py, pz, w [np]).
#include <cstdio>
#include <vector>

#include "mesh_qs.h"

template <class T>
static bool rd(std::FILE* f, T* p, size_t n) {
    return std::fread(p, sizeof(T), n, f) == n;
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: run_step <inputs.bin> <onaxis_out.bin>\n");
        return 2;
    }
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t iv[9];
    double dv[6];
    int64_t nb = 0, np = 0;
    if (!rd(f, iv, 9) || !rd(f, dv, 6) || !rd(f, &nb, 1)) return 3;
    std::vector<int32_t> bi(nb), bj(nb), bk(nb);
    std::vector<double> b[7];
    if (!rd(f, bi.data(), nb) || !rd(f, bj.data(), nb) || !rd(f, bk.data(), nb)) return 3;
    for (auto& v : b) {
        v.resize(nb);
        if (!rd(f, v.data(), nb)) return 3;
    }
    if (!rd(f, &np, 1)) return 3;
    std::vector<int32_t> cell(np);
    std::vector<double> p[6];
    if (!rd(f, cell.data(), np)) return 3;
    for (auto& v : p) {
        v.resize(np);
        if (!rd(f, v.data(), np)) return 3;
    }
    std::fclose(f);
    try {
        MeshQS mesh(iv[0], iv[1], iv[2], dv[0], dv[1], dv[2], dv[3], iv[3], iv[4], iv[5], dv[4],
                    dv[5], iv[6], iv[7]);
        mesh.LoadBeam(nb, bi.data(), bj.data(), bk.data(), b[0].data(), b[1].data(),
                      b[2].data(), b[3].data(), b[4].data(), b[5].data(), b[6].data());
        for (int s = 0; s < iv[8]; s++) {
            mesh.LoadFrontParticles(np, cell.data(), p[0].data(), p[1].data(), p[2].data(),
                                    p[3].data(), p[4].data(), p[5].data());
            mesh.MoveBeamParticles();
            mesh.MoveAllSplitLayers();
        }
        const std::vector<double> ex = mesh.OnAxisEx(iv[2]);
        std::FILE* o = std::fopen(argv[2], "wb");
        if (!o || std::fwrite(ex.data(), sizeof(double), ex.size(), o) != ex.size()) return 4;
        std::fclose(o);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "MeshQS: %s\n", e.what());
        return 1;
    }
    return 0;
}
