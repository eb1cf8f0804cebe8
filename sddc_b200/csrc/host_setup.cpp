// Host-side set-up for the SDDC residual drop-in (declared in sddc_host.h).
//
// Single-rank restatement of the reference host's mesh pipeline:
//   CHECK_MESH     connectivity.f90:237-298   make every cell counter-clockwise
//   CONNECTIVITY   connectivity.f90:1-234     faces, left/right cells, local faces
//   CONNECT_BDRY   connect_bdry.f90:1-354     boundary lists, interior list, cyclic split
//   MAPCYCLOC      map_cyc_loc.f90:1-42       periodic face pairs
//   setsandpoints / computeLandM  initsetup.f90:171-344
//   mapder / calcjacob (bilinear) mapder.f90:1-76, calcjacob.f90:1-132
//   MAPDER_8_NODE / calcjacob (8-node serendipity cells, CURVE_WALL = 1)
//                                mapder.f90:88-253, calcjacob.f90:12-132
//   tecplotter2dsetup            tecplotter2dsetup.f90:1-160  plot mesh
// and the reference's restart and Tecplot file formats (output_format.h).
// The face numbering and the choice of left cell (the lower cell index,
// which visits the face first) follow CONNECTIVITY, because the Rusanov flux
// is evaluated with the left cell's metric and trace first.
// Partitioned runs (MATCHPROC, MATCHCYCREM, processor faces) do not exist on
// one GPU: a face that is neither interior nor on a listed boundary, or a
// cyclic face without a partner, is an error here.

#include "../../include/sddc_host.h"
#include "sd_basis.h"
#include "output_format.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

constexpr double kTolCyc = 1e-5;           // tolCYC, setup2d.f90:62
// IVFACE(IFACE,1:2): local face -> its two local vertices (connectivity.f90:73-83)
constexpr int kIvFace[4][2] = {{1, 2}, {2, 3}, {3, 4}, {4, 1}};

}  // namespace

struct sddc_mesh {
    int ncell = 0, nvert = 0, nface = 0;
    std::vector<int> ivcell;   // (ncell,4), 1-based, CCW
    std::vector<double> xv, yv;
    std::vector<int> ic2f;     // (ncell,4)
    std::vector<int> if2c;     // (nface,4)
    std::vector<int> if2v;     // (nface,2)
    std::vector<int> inter, inl, outl, symp, wall, cycl, freeb, cycloc, cycrem;
    std::vector<int> pair1, pair2;
    int nreversed = 0, nprocint = 0;

    int iv(int c, int k) const { return ivcell[(c - 1) + (size_t)ncell * (k - 1)]; }
    int &iv(int c, int k) { return ivcell[(c - 1) + (size_t)ncell * (k - 1)]; }
};

extern "C" const char *sddc_host_last_error(void) { return g_err.c_str(); }

// ---------------------------------------------------------------- operators

using sddc::lagrange;
using sddc::sd_points;

extern "C" int sddc_sd_operators(int N, double *Xs, double *Xf, double *Lmat, double *Mmat)
{
    if (N < 2 || N > 6) return fail(-1, "sddc_sd_operators: N must be in [2, 6]");
    sd_points(N, Xs, Xf);
    const int N1 = N + 1;
    for (int f = 1; f <= N1; f++)
        for (int s = 1; s <= N; s++) Lmat[(f - 1) + N1 * (s - 1)] = lagrange(Xs, N, s, Xf[f - 1]);
    // derivative of the flux-point basis at the solution points, written as
    // the sum over k of the product rule terms (computeLandM)
    for (int f = 1; f <= N1; f++)
        for (int s = 1; s <= N; s++) {
            const double x = Xs[s - 1];
            double acc = 0.0;
            for (int k = 1; k <= N1; k++) {
                if (k == f) continue;
                double num = 1.0, den = 1.0;
                for (int q = 1; q <= N1; q++) {
                    if (q != f && q != k) num = num * (x - Xf[q - 1]);
                    if (q != f) den = den * (Xf[f - 1] - Xf[q - 1]);
                }
                acc = acc + num / den;
            }
            Mmat[(f - 1) + N1 * (s - 1)] = acc;
        }
    return 0;
}

// ---------------------------------------------------------------- mesh

static int build_mesh(sddc_mesh &m, const int *bnd_v, const int *bnd_type, int nbound,
                      double dxcycl, double dycycl)
{
    const int NC = m.ncell, NVERT = m.nvert;
    // CHECK_MESH: signed shoelace sum; positive means clockwise -> swap 1<->2, 3<->4
    for (int c = 1; c <= NC; c++) {
        double sum = 0.0;
        for (int f = 0; f < 4; f++) {
            int a = m.iv(c, kIvFace[f][0]), b = m.iv(c, kIvFace[f][1]);
            sum += (m.xv[b - 1] - m.xv[a - 1]) * (m.yv[a - 1] + m.yv[b - 1]);
        }
        if (sum > 0) {
            int v1 = m.iv(c, 1), v2 = m.iv(c, 2), v3 = m.iv(c, 3), v4 = m.iv(c, 4);
            m.iv(c, 1) = v2; m.iv(c, 2) = v1; m.iv(c, 3) = v4; m.iv(c, 4) = v3;
            m.nreversed++;
        }
    }
    // vertex -> cells (CSR in cell order)
    std::vector<int> start(NVERT + 2, 0), fillc(NVERT + 1, 0);
    for (int c = 1; c <= NC; c++)
        for (int k = 1; k <= 4; k++) {
            int v = m.iv(c, k);
            if (v < 1 || v > NVERT) return fail(-2, "vertex index out of range in IVCELL");
            fillc[v]++;
        }
    for (int v = 1; v <= NVERT; v++)
        if (fillc[v] == 0) return fail(-3, "vertex " + std::to_string(v) + " belongs to no cell");
    start[1] = 0;
    for (int v = 1; v <= NVERT; v++) start[v + 1] = start[v] + fillc[v];
    std::vector<int> cells(start[NVERT + 1]);
    {
        std::vector<int> pos(start.begin(), start.end());
        for (int c = 1; c <= NC; c++)
            for (int k = 1; k <= 4; k++) cells[pos[m.iv(c, k)]++] = c;
    }
    // CONNECTIVITY: the first cell to visit a face is its left cell
    m.ic2f.assign((size_t)NC * 4, 0);
    std::vector<int> fl, fr, fv1, fv2;
    fl.reserve((size_t)NC * 2 + 8);
    auto ic2f = [&](int c, int f) -> int & { return m.ic2f[(c - 1) + (size_t)NC * (f - 1)]; };
    for (int c = 1; c <= NC; c++) {
        for (int f = 1; f <= 4; f++) {
            if (ic2f(c, f) != 0) continue;
            const int vb = m.iv(c, kIvFace[f - 1][0]), v1 = m.iv(c, kIvFace[f - 1][1]);
            int nb = 0, nbf = 0;
            for (int k = start[vb]; k < start[vb + 1] && !nb; k++) {
                int cc = cells[k];
                if (cc == c) continue;
                for (int ff = 1; ff <= 4; ff++) {
                    int a = m.iv(cc, kIvFace[ff - 1][0]), b = m.iv(cc, kIvFace[ff - 1][1]);
                    if ((vb == a && v1 == b) || (vb == b && v1 == a)) {
                        nb = cc;
                        nbf = ff;
                        break;
                    }
                }
            }
            fl.push_back(c);
            fr.push_back(nb);
            fv1.push_back(vb);
            fv2.push_back(v1);
            const int face = (int)fl.size();
            if (nb) ic2f(nb, nbf) = face;
            ic2f(c, f) = face;
        }
    }
    const int NF = (int)fl.size();
    m.nface = NF;
    m.if2c.assign((size_t)NF * 4, 0);
    m.if2v.assign((size_t)NF * 2, 0);
    auto IF2C = [&](int f, int k) -> int & { return m.if2c[(f - 1) + (size_t)NF * (k - 1)]; };
    for (int f = 1; f <= NF; f++) {
        IF2C(f, 1) = fl[f - 1];
        IF2C(f, 2) = fr[f - 1];
        m.if2v[f - 1] = fv1[f - 1];
        m.if2v[(f - 1) + NF] = fv2[f - 1];
    }
    // local face of the left cell from the face's vertex sequence, and of
    // the right cell from the reversed sequence
    for (int f = 1; f <= NF; f++) {
        const int a = fv1[f - 1], b = fv2[f - 1];
        const int c1 = IF2C(f, 1), c2 = IF2C(f, 2);
        for (int lf = 1; lf <= 4 && !IF2C(f, 3); lf++)
            if (m.iv(c1, kIvFace[lf - 1][0]) == a && m.iv(c1, kIvFace[lf - 1][1]) == b) IF2C(f, 3) = lf;
        if (!IF2C(f, 3)) return fail(-4, "connectivity: face " + std::to_string(f) + " not on its left cell");
        if (c2) {
            for (int lf = 1; lf <= 4 && !IF2C(f, 4); lf++)
                if (m.iv(c2, kIvFace[lf - 1][1]) == a && m.iv(c2, kIvFace[lf - 1][0]) == b) IF2C(f, 4) = lf;
            if (!IF2C(f, 4))
                return fail(-4, "connectivity: face " + std::to_string(f) +
                                    " has the same orientation in both cells");
        }
    }
    // CONNECT_BDRY: attach each boundary record to its face
    std::vector<char> is_bnd(NF + 1, 0);
    for (int ib = 0; ib < nbound; ib++) {
        const int vb1 = bnd_v[ib], vb3 = bnd_v[ib + nbound];
        if (vb1 < 1 || vb1 > NVERT || vb3 < 1 || vb3 > NVERT)
            return fail(-5, "boundary record " + std::to_string(ib + 1) + ": vertex out of range");
        int icc = 0;  // last cell touching both vertices, as the reference's double loop
        for (int k1 = start[vb1]; k1 < start[vb1 + 1]; k1++)
            for (int k3 = start[vb3]; k3 < start[vb3 + 1]; k3++)
                if (cells[k1] == cells[k3]) icc = cells[k1];
        if (!icc) return fail(-5, "boundary record " + std::to_string(ib + 1) + " touches no cell");
        int face = 0;
        for (int lf = 1; lf <= 4; lf++) {
            int a = m.iv(icc, kIvFace[lf - 1][0]), b = m.iv(icc, kIvFace[lf - 1][1]);
            if ((a == vb1 || b == vb1) && (a == vb3 || b == vb3)) {
                face = ic2f(icc, lf);
                break;
            }
        }
        if (!face) return fail(-5, "boundary record " + std::to_string(ib + 1) + " is not a cell face");
        is_bnd[face] = 1;
        switch (bnd_type[ib]) {
        case SDDC_BC_INLE: m.inl.push_back(face); break;
        case SDDC_BC_OUTL: m.outl.push_back(face); break;
        case SDDC_BC_SYMP: m.symp.push_back(face); break;
        case SDDC_BC_WALL: m.wall.push_back(face); break;
        case SDDC_BC_CYCL: m.cycl.push_back(face); break;
        case SDDC_BC_FREE: m.freeb.push_back(face); break;
        default: return fail(-6, "boundary record " + std::to_string(ib + 1) + ": unknown type");
        }
    }
    for (int f = 1; f <= NF; f++) {
        if (IF2C(f, 2) != 0) m.inter.push_back(f);
        else if (!is_bnd[f]) m.nprocint++;
    }
    if (m.nprocint)
        return fail(-7, std::to_string(m.nprocint) +
                            " boundary faces carry no boundary condition (processor faces do not "
                            "exist on one GPU)");
    // cyclic faces: local when a translated partner exists (connect_bdry.f90:281-308)
    auto mid = [&](int f, double &x, double &y) {
        int a = m.if2v[f - 1], b = m.if2v[(f - 1) + NF];
        x = (m.xv[a - 1] + m.xv[b - 1]) / 2;
        y = (m.yv[a - 1] + m.yv[b - 1]) / 2;
    };
    auto matches = [&](int f1, int f2) {
        double x1, y1, x2, y2;
        mid(f1, x1, y1);
        mid(f2, x2, y2);
        double ex = std::fabs(std::fabs(x1 - x2) - dxcycl), ey = std::fabs(std::fabs(y1 - y2) - dycycl);
        return (std::fabs(x1 - x2) < kTolCyc && ey < kTolCyc) || (std::fabs(y1 - y2) < kTolCyc && ex < kTolCyc);
    };
    for (int f : m.cycl) {
        bool found = false;
        for (int g : m.cycl)
            if (matches(f, g)) { found = true; break; }
        (found ? m.cycloc : m.cycrem).push_back(f);
    }
    if (!m.cycrem.empty())
        return fail(-8, std::to_string(m.cycrem.size()) + " cyclic faces have no periodic partner");
    // MAPCYCLOC: pair each local cyclic face with a later one
    for (size_t i = 0; i < m.cycloc.size(); i++)
        for (size_t j = i + 1; j < m.cycloc.size(); j++)
            if (matches(m.cycloc[i], m.cycloc[j])) {
                m.pair1.push_back(m.cycloc[i]);
                m.pair2.push_back(m.cycloc[j]);
            }
    if (m.pair1.size() * 2 != m.cycloc.size())
        return fail(-9, "cyclic faces do not pair up (" + std::to_string(m.pair1.size()) + " pairs for " +
                            std::to_string(m.cycloc.size()) + " faces)");
    return 0;
}

extern "C" int sddc_mesh_build(sddc_mesh **out, int ncell, int nvert, const int *ivcell, const double *xv,
                               const double *yv, int nbound, const int *bnd_v, const int *bnd_type,
                               double dxcycl, double dycycl)
{
    if (!out) return fail(-1, "sddc_mesh_build: out is NULL");
    *out = nullptr;
    if (ncell < 1 || nvert < 4 || !ivcell || !xv || !yv || nbound < 0 || (nbound && (!bnd_v || !bnd_type)))
        return fail(-1, "sddc_mesh_build: bad arguments");
    auto *m = new sddc_mesh();
    m->ncell = ncell;
    m->nvert = nvert;
    m->ivcell.assign(ivcell, ivcell + (size_t)ncell * 4);
    m->xv.assign(xv, xv + nvert);
    m->yv.assign(yv, yv + nvert);
    int rc = build_mesh(*m, bnd_v, bnd_type, nbound, dxcycl, dycycl);
    if (rc) {
        delete m;
        return rc;
    }
    *out = m;
    return 0;
}

extern "C" void sddc_mesh_destroy(sddc_mesh *m) { delete m; }

extern "C" int sddc_mesh_counts(const sddc_mesh *m, int *c)
{
    if (!m || !c) return fail(-1, "sddc_mesh_counts: NULL argument");
    c[SDDC_MC_NFACE] = m->nface;
    c[SDDC_MC_NINTER] = (int)m->inter.size();
    c[SDDC_MC_NINLET] = (int)m->inl.size();
    c[SDDC_MC_NOUTLET] = (int)m->outl.size();
    c[SDDC_MC_NSYMP] = (int)m->symp.size();
    c[SDDC_MC_NWALL] = (int)m->wall.size();
    c[SDDC_MC_NCYCL] = (int)m->cycl.size();
    c[SDDC_MC_NCYCLOC] = (int)m->cycloc.size();
    c[SDDC_MC_NCYCREM] = (int)m->cycrem.size();
    c[SDDC_MC_NPAIR] = (int)m->pair1.size();
    c[SDDC_MC_NPROCINT] = m->nprocint;
    c[SDDC_MC_NFREE] = (int)m->freeb.size();
    c[SDDC_MC_NREVERSED] = m->nreversed;
    c[SDDC_MC_NVERT] = m->nvert;
    c[SDDC_MC_NCELL] = m->ncell;
    return 0;
}

static void copy_list(const std::vector<int> &v, int *dst)
{
    if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(int) * v.size());
}

extern "C" int sddc_mesh_tables(const sddc_mesh *m, int *if2c, int *if2v, int *ibfinter, int *ibfinl,
                                int *ibfout, int *ibfwal, int *ibfsymp, int *ibfree, int *cyc2fpair,
                                int *ivcell_ccw)
{
    if (!m) return fail(-1, "sddc_mesh_tables: NULL mesh");
    copy_list(m->if2c, if2c);
    copy_list(m->if2v, if2v);
    copy_list(m->inter, ibfinter);
    copy_list(m->inl, ibfinl);
    copy_list(m->outl, ibfout);
    copy_list(m->wall, ibfwal);
    copy_list(m->symp, ibfsymp);
    copy_list(m->freeb, ibfree);
    copy_list(m->ivcell, ivcell_ccw);
    if (cyc2fpair) {
        const size_t np = m->pair1.size();
        for (size_t i = 0; i < np; i++) {
            cyc2fpair[i] = m->pair1[i];
            cyc2fpair[i + np] = m->pair2[i];
        }
    }
    return 0;
}

// ---------------------------------------------------------------- metrics

// derivatives of the four bilinear shape functions at (psi, eta) (mapder)
static void shape_derivs(double psi, double eta, double d[4][2])
{
    d[0][0] = eta - 1.0; d[0][1] = psi - 1.0;
    d[1][0] = 1.0 - eta; d[1][1] = -psi;
    d[2][0] = eta;       d[2][1] = psi;
    d[3][0] = -eta;      d[3][1] = 1.0 - psi;
}

struct Derivs {
    double xpsi, ypsi, xeta, yeta;
};

static Derivs map_derivs(const double X[4], const double Y[4], double psi, double eta)
{
    double d[4][2];
    shape_derivs(psi, eta, d);
    Derivs r{0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < 4; k++) {
        r.xpsi = r.xpsi + d[k][0] * X[k];
        r.ypsi = r.ypsi + d[k][0] * Y[k];
        r.xeta = r.xeta + d[k][1] * X[k];
        r.yeta = r.yeta + d[k][1] * Y[k];
    }
    return r;
}

extern "C" int sddc_mesh_metrics(const sddc_mesh *m, int N, double *S1, double *S2, double *Jac, double *xxsolu)
{
    if (!m) return fail(-1, "sddc_mesh_metrics: NULL mesh");
    if (N < 2 || N > 6) return fail(-1, "sddc_mesh_metrics: N must be in [2, 6]");
    double Xs[8], Xf[8];
    sd_points(N, Xs, Xf);
    const int N1 = N + 1;
    for (int c = 1; c <= m->ncell; c++) {
        double X[4], Y[4];
        for (int k = 1; k <= 4; k++) {
            X[k - 1] = m->xv[m->iv(c, k) - 1];
            Y[k - 1] = m->yv[m->iv(c, k) - 1];
        }
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N; i++) {
                Derivs d = map_derivs(X, Y, Xs[i - 1], Xs[j - 1]);
                if (Jac) Jac[(i - 1) + (size_t)N * ((j - 1) + (size_t)N * (c - 1))] = d.xpsi * d.yeta - d.xeta * d.ypsi;
                if (xxsolu) {
                    // xyCoor_atGps with MapBaseFunc (mapder.f90:79-87, 255-273)
                    const double xi = Xs[i - 1], et = Xs[j - 1];
                    const double fn[4] = {(1.0 - xi) * (1.0 - et), (1.0 - et) * xi, xi * et, (1.0 - xi) * et};
                    double px = 0.0, py = 0.0;
                    for (int k = 0; k < 4; k++) {
                        px = px + X[k] * fn[k];
                        py = py + Y[k] * fn[k];
                    }
                    size_t b = 2 * ((i - 1) + (size_t)N * ((j - 1) + (size_t)N * (c - 1)));
                    xxsolu[b] = px;
                    xxsolu[b + 1] = py;
                }
            }
        if (S1)
            for (int j = 1; j <= N; j++)
                for (int f = 1; f <= N1; f++) {
                    Derivs d = map_derivs(X, Y, Xf[f - 1], Xs[j - 1]);
                    size_t b = 4 * ((f - 1) + (size_t)N1 * ((j - 1) + (size_t)N * (c - 1)));
                    S1[b + 0] = d.yeta;   // S1(1,1)
                    S1[b + 1] = -d.ypsi;  // S1(2,1)
                    S1[b + 2] = -d.xeta;  // S1(1,2)
                    S1[b + 3] = d.xpsi;   // S1(2,2)
                }
        if (S2)
            for (int f = 1; f <= N1; f++)
                for (int i = 1; i <= N; i++) {
                    Derivs d = map_derivs(X, Y, Xs[i - 1], Xf[f - 1]);
                    size_t b = 4 * ((i - 1) + (size_t)N * ((f - 1) + (size_t)N1 * (c - 1)));
                    S2[b + 0] = d.yeta;
                    S2[b + 1] = -d.ypsi;
                    S2[b + 2] = -d.xeta;
                    S2[b + 3] = d.xpsi;
                }
    }
    return 0;
}

// ---------------------------------------------------------------- 8-node cells

// derivatives of the eight serendipity shape functions at (psi, eta)
// (MAPDER_8_NODE, mapder.f90:117-253; nodes 1-4 the corners counter-
// clockwise, 5-8 the mid-side nodes of edges 1-2, 2-3, 3-4, 4-1)
static void shape_derivs8(double psi, double eta, double d[8][2])
{
    d[0][0] = (1.0 - eta) * (4.0 * psi + 2.0 * eta - 3.0);
    d[0][1] = (1.0 - psi) * (4.0 * eta + 2.0 * psi - 3.0);
    d[1][0] = (1.0 - eta) * (4.0 * psi - 2.0 * eta - 1.0);
    d[1][1] = psi * (4.0 * eta - 2.0 * psi - 1.0);
    d[2][0] = eta * (4.0 * psi + 2.0 * eta - 3.0);
    d[2][1] = psi * (4.0 * eta + 2.0 * psi - 3.0);
    d[3][0] = eta * (4.0 * psi - 2.0 * eta - 1.0);
    d[3][1] = (1.0 - psi) * (4.0 * eta - 2.0 * psi - 1.0);
    d[4][0] = 4.0 * (1.0 - eta) * (1.0 - 2.0 * psi);
    d[4][1] = 4.0 * psi * (psi - 1.0);
    d[5][0] = 4.0 * eta * (1.0 - eta);
    d[5][1] = 4.0 * psi * (1.0 - 2.0 * eta);
    d[6][0] = 4.0 * eta * (1.0 - 2.0 * psi);
    d[6][1] = 4.0 * psi * (1.0 - psi);
    d[7][0] = 4.0 * eta * (eta - 1.0);
    d[7][1] = 4.0 * (1.0 - psi) * (1.0 - 2.0 * eta);
}

// calcjacob's CURVE_WALL = 1 sums, k = 1..8 in order (calcjacob.f90:47-52)
static Derivs map_derivs8(const double *xx, double psi, double eta)
{
    double d[8][2];
    shape_derivs8(psi, eta, d);
    Derivs r{0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < 8; k++) {
        r.xpsi = r.xpsi + d[k][0] * xx[2 * k];
        r.ypsi = r.ypsi + d[k][0] * xx[2 * k + 1];
        r.xeta = r.xeta + d[k][1] * xx[2 * k];
        r.yeta = r.yeta + d[k][1] * xx[2 * k + 1];
    }
    return r;
}

// xyCoor_atGps with MapBaseFunc8 (mapder.f90:91-103, 255-273)
static void serendipity_point(const double *xx, double xi, double eta, double &px, double &py)
{
    const double f[8] = {(1.0 - xi) * (1.0 - eta) * (-2.0 * xi - 2.0 * eta + 1.0),
                         xi * (1.0 - eta) * (2.0 * xi - 2.0 * eta - 1.0),
                         xi * eta * (2.0 * xi + 2.0 * eta - 3.0),
                         (1.0 - xi) * eta * (-2.0 * xi + 2.0 * eta - 1.0),
                         4.0 * (1.0 - eta) * (1.0 - xi) * xi,
                         4.0 * eta * (1.0 - eta) * xi,
                         4.0 * (1.0 - xi) * xi * eta,
                         4.0 * (1.0 - eta) * (1.0 - xi) * eta};
    px = 0.0;
    py = 0.0;
    for (int k = 0; k < 8; k++) {
        px = px + xx[2 * k] * f[k];
        py = py + xx[2 * k + 1] * f[k];
    }
}

extern "C" int sddc_metrics8(int N, int ncell, const double *xxf_cell, double *S1, double *S2, double *Jac,
                             double *xxsolu)
{
    if (N < 2 || N > 6) return fail(-1, "sddc_metrics8: N must be in [2, 6]");
    if (ncell < 1 || !xxf_cell) return fail(-1, "sddc_metrics8: bad arguments");
    double Xs[8], Xf[8];
    sd_points(N, Xs, Xf);
    const int N1 = N + 1;
    for (int c = 0; c < ncell; c++) {
        const double *xx = xxf_cell + 16 * (size_t)c;  // xxf_cell(2,8,NCELL)
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N; i++) {
                const size_t ip = (i - 1) + (size_t)N * ((j - 1) + (size_t)N * c);
                if (Jac) {
                    Derivs d = map_derivs8(xx, Xs[i - 1], Xs[j - 1]);
                    Jac[ip] = d.xpsi * d.yeta - d.xeta * d.ypsi;
                }
                if (xxsolu) serendipity_point(xx, Xs[i - 1], Xs[j - 1], xxsolu[2 * ip], xxsolu[2 * ip + 1]);
            }
        if (S1)
            for (int j = 1; j <= N; j++)
                for (int f = 1; f <= N1; f++) {
                    Derivs d = map_derivs8(xx, Xf[f - 1], Xs[j - 1]);
                    size_t b = 4 * ((f - 1) + (size_t)N1 * ((j - 1) + (size_t)N * c));
                    S1[b + 0] = d.yeta;
                    S1[b + 1] = -d.ypsi;
                    S1[b + 2] = -d.xeta;
                    S1[b + 3] = d.xpsi;
                }
        if (S2)
            for (int f = 1; f <= N1; f++)
                for (int i = 1; i <= N; i++) {
                    Derivs d = map_derivs8(xx, Xs[i - 1], Xf[f - 1]);
                    size_t b = 4 * ((i - 1) + (size_t)N * ((f - 1) + (size_t)N1 * c));
                    S2[b + 0] = d.yeta;
                    S2[b + 1] = -d.ypsi;
                    S2[b + 2] = -d.xeta;
                    S2[b + 3] = d.xpsi;
                }
    }
    return 0;
}

// ---------------------------------------------------------------- plot mesh

struct sddc_plotmesh {
    int nre = 0, ncell = 0, plotnodes = 0, plotcells = 0;
    std::vector<double> plotx;  // (2,plotnodes)
    std::vector<int> gnumnode;  // (nre+1,nre+1,ncell)
    std::vector<int> gfac;      // (plotnodes)
    std::vector<int> connec;    // (4,plotcells)
};

// xyCoor_atGps with the bilinear MapBaseFunc (mapder.f90:79-87, 255-273)
static void bilinear_point(const double X[4], const double Y[4], double xi, double et, double &px, double &py)
{
    const double fn[4] = {(1.0 - xi) * (1.0 - et), (1.0 - et) * xi, xi * et, (1.0 - xi) * et};
    px = 0.0;
    py = 0.0;
    for (int k = 0; k < 4; k++) {
        px = px + X[k] * fn[k];
        py = py + Y[k] * fn[k];
    }
}

extern "C" int sddc_plotmesh_build(sddc_plotmesh **out, const sddc_mesh *m, int nre, const double *xxf_cell)
{
    if (!out) return fail(-1, "sddc_plotmesh_build: out is NULL");
    *out = nullptr;
    if (!m) return fail(-1, "sddc_plotmesh_build: NULL mesh");
    if (nre < 1 || nre > 64) return fail(-1, "sddc_plotmesh_build: nre must be in [1, 64]");
    const int Np = nre, n1 = nre + 1, nc = m->ncell;
    const size_t cap = (size_t)n1 * n1 * nc;  // allocate_plot_memory
    if (cap >= (size_t)1 << 31 || (size_t)m->nvert > cap) return fail(-1, "sddc_plotmesh_build: mesh too large");
    const double tolplot = 1e-5;
    auto pm = std::make_unique<sddc_plotmesh>();
    pm->nre = nre;
    pm->ncell = nc;
    std::vector<double> px(2 * cap);
    std::vector<int> gfac(cap, 0), isfacenod(m->nface + 1, 0), gfacenode((size_t)(Np > 1 ? Np - 1 : 1) * (m->nface + 1));
    pm->gnumnode.assign(cap, 0);
    auto gn = [&](int ii, int jj, int c) -> int & {
        return pm->gnumnode[(ii - 1) + (size_t)n1 * ((jj - 1) + (size_t)n1 * (c - 1))];
    };
    int plotnodes = 0, plotcells = 0;
    // the four vertices of each cell: plot nodes 1..NVERT are the vertices
    for (int c = 1; c <= nc; c++) {
        const int v[4] = {m->iv(c, 1), m->iv(c, 2), m->iv(c, 3), m->iv(c, 4)};
        gn(1, 1, c) = v[0];
        gn(Np + 1, 1, c) = v[1];
        gn(Np + 1, Np + 1, c) = v[2];
        gn(1, Np + 1, c) = v[3];
        for (int k = 0; k < 4; k++) {
            const int g = v[k];
            if (gfac[g - 1] == 0) {
                plotnodes++;
                px[2 * (g - 1)] = m->xv[g - 1];
                px[2 * (g - 1) + 1] = m->yv[g - 1];
            }
            gfac[g - 1]++;
        }
    }
    if (plotnodes != m->nvert)
        return fail(-1, "sddc_plotmesh_build: " + std::to_string(m->nvert - plotnodes) +
                            " vertices belong to no cell (the plot node numbering needs every vertex)");
    std::vector<int> connec(4 * (size_t)Np * Np * nc);
    for (int c = 1; c <= nc; c++) {
        double X[4], Y[4];
        for (int k = 1; k <= 4; k++) {
            X[k - 1] = m->xv[m->iv(c, k) - 1];
            Y[k - 1] = m->yv[m->iv(c, k) - 1];
        }
        // the cell's map: bilinear, or the eight nodes of xxf_cell
        const double *xx8 = xxf_cell ? xxf_cell + 16 * (size_t)(c - 1) : nullptr;
        auto point = [&](double xi, double et, double &px_, double &py_) {
            if (xx8) serendipity_point(xx8, xi, et, px_, py_);
            else bilinear_point(X, Y, xi, et, px_, py_);
        };
        // the inner nodes of the four faces, counter-clockwise
        for (int k = 1; k <= 4; k++) {
            const int iface = m->ic2f[(c - 1) + (size_t)nc * (k - 1)];
            for (int en = 1; en <= Np - 1; en++) {
                int ii = 0, jj = 0;
                switch (k) {
                case 1: ii = en + 1; jj = 1; break;
                case 2: ii = Np + 1; jj = en + 1; break;
                case 3: ii = Np + 1 - en; jj = Np + 1; break;
                default: ii = 1; jj = Np + 1 - en; break;
                }
                const double xsi = (double)(ii - 1) / (double)Np, eta = (double)(jj - 1) / (double)Np;
                double rx, ry;
                point(xsi, eta, rx, ry);
                if (isfacenod[iface] == 1) {
                    bool match = false;
                    for (int e = 1; e <= Np - 1; e++) {
                        const int g = gfacenode[(e - 1) + (size_t)(Np - 1) * iface];
                        const double dx = rx - px[2 * (g - 1)], dy = ry - px[2 * (g - 1) + 1];
                        if (std::fabs(std::sqrt(dx * dx + dy * dy)) <= tolplot) {
                            gn(ii, jj, c) = g;
                            gfac[g - 1]++;
                            match = true;
                        }
                    }
                    if (!match)
                        return fail(-1, "sddc_plotmesh_build: face " + std::to_string(iface) + " node of cell " +
                                            std::to_string(c) + " matches none of the face's plot nodes");
                } else {
                    plotnodes++;
                    px[2 * (plotnodes - 1)] = rx;
                    px[2 * (plotnodes - 1) + 1] = ry;
                    gn(ii, jj, c) = plotnodes;
                    gfacenode[(en - 1) + (size_t)(Np - 1) * iface] = plotnodes;
                    gfac[plotnodes - 1]++;
                }
            }
            if (isfacenod[iface] == 0) isfacenod[iface] = 1;
        }
        // interior nodes
        for (int ii = 2; ii <= Np; ii++)
            for (int jj = 2; jj <= Np; jj++) {
                double rx, ry;
                point((double)(ii - 1) / (double)Np, (double)(jj - 1) / (double)Np, rx, ry);
                plotnodes++;
                px[2 * (plotnodes - 1)] = rx;
                px[2 * (plotnodes - 1) + 1] = ry;
                gn(ii, jj, c) = plotnodes;
                gfac[plotnodes - 1]++;
            }
        // plot cells
        for (int ii = 1; ii <= Np; ii++)
            for (int jj = 1; jj <= Np; jj++) {
                int *q = &connec[4 * (size_t)plotcells];
                q[0] = gn(ii, jj, c);
                q[1] = gn(ii + 1, jj, c);
                q[2] = gn(ii + 1, jj + 1, c);
                q[3] = gn(ii, jj + 1, c);
                plotcells++;
            }
    }
    pm->plotnodes = plotnodes;
    pm->plotcells = plotcells;
    px.resize(2 * (size_t)plotnodes);
    gfac.resize(plotnodes);
    pm->plotx = std::move(px);
    pm->gfac = std::move(gfac);
    pm->connec = std::move(connec);
    *out = pm.release();
    return 0;
}

extern "C" void sddc_plotmesh_destroy(sddc_plotmesh *pm) { delete pm; }

extern "C" int sddc_plotmesh_counts(const sddc_plotmesh *pm, int *plotnodes, int *plotcells)
{
    if (!pm) return fail(-1, "sddc_plotmesh_counts: NULL plot mesh");
    if (plotnodes) *plotnodes = pm->plotnodes;
    if (plotcells) *plotcells = pm->plotcells;
    return 0;
}

extern "C" int sddc_plotmesh_tables(const sddc_plotmesh *pm, double *plotx, int *gnumnode, int *gnode_factor,
                                    int *connec)
{
    if (!pm) return fail(-1, "sddc_plotmesh_tables: NULL plot mesh");
    if (plotx) std::memcpy(plotx, pm->plotx.data(), pm->plotx.size() * sizeof(double));
    copy_list(pm->gnumnode, gnumnode);
    copy_list(pm->gfac, gnode_factor);
    copy_list(pm->connec, connec);
    return 0;
}

// ---------------------------------------------------------------- output files

static int copy_name(const std::string &s, char *buf, int len)
{
    if (!buf || len <= (int)s.size()) return fail(-1, "file name buffer too short");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return (int)s.size();
}

extern "C" int sddc_restart_filename(int iter, char *buf, int len)
{
    return copy_name(sddc::fmt::restart_name(iter), buf, len);
}

extern "C" int sddc_tecplot_filename(double ctime, char *buf, int len)
{
    return copy_name(sddc::fmt::tecplot_name(ctime), buf, len);
}

extern "C" int sddc_restart_write(const char *path, int iter, double ctime, int N, int ncell, const int *icg,
                                  const double *Q)
{
    if (!path || !Q || N < 2 || N > 6 || ncell < 1) return fail(-1, "sddc_restart_write: bad arguments");
    std::string err;
    return sddc::fmt::write_restart(path, iter, ctime, N, ncell, icg, Q, err) ? fail(-1, err) : 0;
}

extern "C" int sddc_restart_read(const char *path, int N, int ncell, int nrec, const int *icg2ic, int nglob,
                                 double *Q, int *iter, double *ctime)
{
    if (!path || !Q || N < 2 || N > 6 || ncell < 1 || nrec < 0 || (icg2ic && nglob < 1))
        return fail(-1, "sddc_restart_read: bad arguments");
    std::string err;
    return sddc::fmt::read_restart(path, N, ncell, nrec ? nrec : ncell, icg2ic, nglob, Q, iter, ctime, err)
               ? fail(-1, err)
               : 0;
}

extern "C" int sddc_tecplot_write(const char *path, double ctime, int plotnodes, int plotcells, const double *plotx,
                                  const double *plotq, const double *plotav, const int *connec)
{
    if (!path || plotnodes < 1 || plotcells < 1 || !plotx || !plotq || !connec)
        return fail(-1, "sddc_tecplot_write: bad arguments");
    std::vector<double> zeros;
    if (!plotav) zeros.assign(2 * (size_t)plotnodes, 0.0);
    const double *av = plotav ? plotav : zeros.data();
    sddc::fmt::PlotVar vars[sddc::fmt::kPlotVars] = {{plotx, 2}, {plotx + 1, 2}};
    for (int v = 0; v < 9; v++) vars[2 + v] = {plotq + v, 9};
    vars[11] = {av, 2};
    vars[12] = {av + 1, 2};
    std::string err;
    return sddc::fmt::write_tecplot(path, ctime, plotnodes, plotcells, vars, connec, err) ? fail(-1, err) : 0;
}
