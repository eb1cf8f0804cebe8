// Host-side packing of the reference's set-up tables (module setup2d,
// setup2d.f90:39-102, Fortran layout, 1-based lists) into the two device
// records every stage launch reads: the per-cell metric record (MetLayout in
// stage_kernel.cuh) and the (cell, local face) records.  sddc_set_tables and
// sddc_noalloc_pack_tables both build their records here, so the two entry
// points cannot drift apart.
#pragma once

#include <cstddef>
#include <cstring>
#include <string>

#include "stage_kernel.cuh"

namespace sddc {

// doubles per cell of the packed metric record
inline int met_record_doubles(int N)
{
    switch (N) {
    case 2: return MetLayout<2>::kSize;
    case 3: return MetLayout<3>::kSize;
    case 4: return MetLayout<4>::kSize;
    case 5: return MetLayout<5>::kSize;
    default: return MetLayout<6>::kSize;
    }
}

// met[c * met_record_doubles(N) + ...]: S1(1,1:2,r,j) at the xi flux points
// (MetLayout::normal(0, j, r)), S2(2,1:2,i,r) at the eta flux points
// (normal(1, i, r)), then Jac(i,j) at kJac + i + N*j; the padding is zero
inline void pack_metric_records(int N, int ncell, const double *S1, const double *S2, const double *Jac, double *met)
{
    const int N1 = N + 1, msize = met_record_doubles(N), kFam = 2 * N * N1, kJac = 2 * kFam;
    std::memset(met, 0, (size_t)ncell * msize * sizeof(double));
    for (size_t c = 0; c < (size_t)ncell; c++) {
        double *m = met + c * msize;
        for (int j = 0; j < N; j++)
            for (int r = 0; r < N1; r++) {
                const size_t b = 4 * (r + (size_t)N1 * (j + (size_t)N * c));
                m[2 * (j * N1 + r)] = S1[b + 0];      // S1(1,1,r,j)
                m[2 * (j * N1 + r) + 1] = S1[b + 2];  // S1(1,2,r,j)
            }
        for (int i = 0; i < N; i++)
            for (int r = 0; r < N1; r++) {
                const size_t b = 4 * (i + (size_t)N * (r + (size_t)N1 * c));
                m[kFam + 2 * (i * N1 + r)] = S2[b + 1];      // S2(2,1,i,r)
                m[kFam + 2 * (i * N1 + r) + 1] = S2[b + 3];  // S2(2,2,i,r)
            }
        for (int k = 0; k < N * N; k++) m[kJac + k] = Jac[k + (size_t)N * N * c];
    }
}

// The face lists the reference's set-up builds, as the tables it names:
// IF2C(NFACE,4) (left cell, right cell, their local faces;
// connectivity.f90:98-216), IBFINTER and the boundary lists (INLE, OUTL,
// WALL, SYMP, FREE; connect_bdry.f90:187-221) and CYC2FPAIR(NPAIR,2)
// (map_cyc_loc.f90:9-40).
struct FaceLists {
    const int *IF2C;
    int nface;
    const int *ibfinter;
    int ninter;
    const int *ibfinl;
    int ninlet;
    const int *ibfout;
    int noutlet;
    const int *ibfwal;
    int nwall;
    const int *ibfsymp;
    int nsymp;
    const int *ibfree;
    int nfree;
    const int *cyc2fpair;
    int npair;
    // processor faces of a decomposed run (IBFPROC, in exchange-slot order;
    // IF2C(K,1) and IF2C(K,3) are the own cell and its local face)
    const int *ibfproc = nullptr;
    int nproc = 0;
};

// rec[2 * (cell * 4 + lf - 1) + {0, 1}] (cell 0-based): the partner cell
// (0-based; -1 on a boundary; the exchange slot of a processor face) and
// kind | partner's local face << 8.  A shared face (interior or cyclic pair)
// gives its left cell (IF2C(:,1), the first face of a pair) kind kFaceLeft
// and the other kFaceRight.  Returns "" or what is wrong with the lists (an
// entry out of range, a (cell, local face) listed twice or in no list).
inline std::string build_face_records(int ncell, const FaceLists &fl, int *rec)
{
    for (size_t k = 0; k < (size_t)ncell * 4; k++) {
        rec[2 * k] = -1;
        rec[2 * k + 1] = kFaceNone;
    }
    const int nface = fl.nface;
    auto IF2 = [&](int f, int k) { return fl.IF2C[(f - 1) + (size_t)nface * (k - 1)]; };
    std::string msg;
    auto claim = [&](int cell, int lf, int partner, int kind, int plf) {
        if (cell < 1 || cell > ncell || lf < 1 || lf > 4 || (partner && (partner < 1 || partner > ncell)) ||
            (partner && (plf < 1 || plf > 4))) {
            if (msg.empty()) msg = "face list entry out of range";
            return;
        }
        int *r = rec + 2 * ((size_t)(cell - 1) * 4 + (lf - 1));
        if ((r[1] & 0xff) != kFaceNone) {
            if (msg.empty())
                msg = "cell " + std::to_string(cell) + " local face " + std::to_string(lf) + " is listed twice";
            return;
        }
        r[0] = partner ? partner - 1 : -1;
        r[1] = kind | (plf << 8);
    };
    auto face_ok = [&](int f) { return f >= 1 && f <= nface; };
    for (int k = 0; k < fl.ninter && msg.empty(); k++) {
        const int f = fl.ibfinter[k];
        if (!face_ok(f)) { msg = "IBFINTER entry out of range"; break; }
        claim(IF2(f, 1), IF2(f, 3), IF2(f, 2), kFaceLeft, IF2(f, 4));
        claim(IF2(f, 2), IF2(f, 4), IF2(f, 1), kFaceRight, IF2(f, 3));
    }
    for (int k = 0; k < fl.npair && msg.empty(); k++) {
        const int f1 = fl.cyc2fpair[k], f2 = fl.cyc2fpair[k + fl.npair];
        if (!face_ok(f1) || !face_ok(f2)) { msg = "CYC2FPAIR entry out of range"; break; }
        claim(IF2(f1, 1), IF2(f1, 3), IF2(f2, 1), kFaceLeft, IF2(f2, 3));
        claim(IF2(f2, 1), IF2(f2, 3), IF2(f1, 1), kFaceRight, IF2(f1, 3));
    }
    const int *lists[5] = {fl.ibfinl, fl.ibfout, fl.ibfwal, fl.ibfsymp, fl.ibfree};
    const int counts[5] = {fl.ninlet, fl.noutlet, fl.nwall, fl.nsymp, fl.nfree};
    const int kinds[5] = {kFaceInle, kFaceOutl, kFaceWall, kFaceSymp, kFaceFree};
    for (int t = 0; t < 5 && msg.empty(); t++)
        for (int k = 0; k < counts[t]; k++) {
            const int f = lists[t][k];
            if (!face_ok(f)) { msg = "boundary list entry out of range"; break; }
            claim(IF2(f, 1), IF2(f, 3), 0, kinds[t], 0);
        }
    for (int b = 0; b < fl.nproc && msg.empty(); b++) {
        const int f = fl.ibfproc[b];
        if (!face_ok(f)) { msg = "IBFPROC entry out of range"; break; }
        const int cell = IF2(f, 1), lf = IF2(f, 3);
        claim(cell, lf, 0, kFaceProc, 0);
        if (msg.empty()) rec[2 * ((size_t)(cell - 1) * 4 + (lf - 1))] = b;
    }
    if (msg.empty())
        for (size_t k = 0; k < (size_t)ncell * 4; k++)
            if ((rec[2 * k + 1] & 0xff) == kFaceNone) {
                msg = "cell " + std::to_string(k / 4 + 1) + " local face " + std::to_string(k % 4 + 1) +
                      " is in no face list (a face whose other cell is on another rank is a processor face, "
                      "sddc_set_proc_faces)";
                break;
            }
    return msg;
}

}  // namespace sddc
