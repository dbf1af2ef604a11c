// host_geom.h -- host-side geometry for the engine: unit cell, k^2 table,
// stress weights, contour discretisation, FFT plans.  Plain C++ (runs on
// the CPU at setup and after each cell update); make_unit_cell is also
// compiled for the device, where the graph-driven Anderson iteration
// updates the cell.
#pragma once
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/pscf_gpu.h"

#ifdef __CUDACC__
#define PSCFG_HD __host__ __device__
#else
#define PSCFG_HD
#endif

namespace pscfg {

// Contour grid of one chain (src/chain_mod.f90:136-158).  bgn is 0-based:
// block b spans slices bgn[b] .. bgn[b+1].
inline int chain_grid(int nblk, const double *blen, double ds, int *bgn, double *bds)
{
    int s = 0;
    bgn[0] = 0;
    for (int i = 0; i < nblk; i++) {
        int iblk = (int)(blen[i] / ds / 2.0 + 0.5);
        if (iblk == 0) {
            iblk = 1;
            bds[i] = blen[i] / 2.0;
        } else {
            bds[i] = blen[i] / (double)iblk / 2.0;
        }
        s += 2 * iblk;
        bgn[i + 1] = s;
    }
    return s;
}

// Anderson mixing parameter lambda = 1 - 0.9^k of iteration k of the ramp
// (src/iterate_mod.fp.f90:1147-1153), the power by repeated multiplication
// so that host and device agree to the bit.
PSCFG_HD inline double am_lambda_ramp(int k)
{
    double p = 1.0;
    for (int j = 0; j < k; j++) p *= 0.9;
    return 1.0 - p;
}

struct Cell {
    int dim = 1;
    int ncp = 0;
    double G[3][3] = {{0}};
    double dGG[PSCFG_MAXCP][3][3] = {{{0}}};
};

// make_unit_cell + make_G_basis (src/unit_cell_mod.f90:309-664, 723-757).
// Returns false for an unknown crystal system.
PSCFG_HD inline bool make_unit_cell(int dim, int sys, const double *cp, Cell &c)
{
    double R[3][3] = {{0}}, dR[3][3][PSCFG_MAXCP];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < PSCFG_MAXCP; k++) dR[i][j][k] = 0.0;
    int ncp = 0;
    const double s75 = sqrt(0.75);
    switch (sys) {
    case PSCFG_LAMELLAR: ncp = 1; R[0][0] = cp[0]; dR[0][0][0] = 1; break;
    case PSCFG_SQUARE: ncp = 1; R[0][0] = R[1][1] = cp[0]; dR[0][0][0] = dR[1][1][0] = 1; break;
    case PSCFG_RECTANGULAR: ncp = 2; R[0][0] = cp[0]; R[1][1] = cp[1]; dR[0][0][0] = dR[1][1][1] = 1; break;
    case PSCFG_HEXAGONAL2D:
        ncp = 1; R[0][0] = cp[0]; R[1][0] = -0.5 * cp[0]; R[1][1] = cp[0] * s75;
        dR[0][0][0] = 1; dR[1][0][0] = -0.5; dR[1][1][0] = s75; break;
    case PSCFG_OBLIQUE:
        // dR(1,1,1) = a as written in src/unit_cell_mod.f90:630
        ncp = 3; R[0][0] = cp[0]; R[1][0] = cp[1] * cos(cp[2]); R[1][1] = cp[1] * sin(cp[2]);
        dR[0][0][0] = cp[0]; dR[1][0][1] = cos(cp[2]); dR[1][1][1] = sin(cp[2]);
        dR[1][0][2] = -cp[1] * sin(cp[2]); dR[1][1][2] = cp[1] * cos(cp[2]); break;
    case PSCFG_CUBIC: ncp = 1; R[0][0] = R[1][1] = R[2][2] = cp[0]; dR[0][0][0] = dR[1][1][0] = dR[2][2][0] = 1; break;
    case PSCFG_TETRAGONAL:
        ncp = 2; R[0][0] = R[1][1] = cp[0]; R[2][2] = cp[1]; dR[0][0][0] = dR[1][1][0] = 1; dR[2][2][1] = 1; break;
    case PSCFG_ORTHORHOMBIC:
        ncp = 3; R[0][0] = cp[0]; R[1][1] = cp[1]; R[2][2] = cp[2]; dR[0][0][0] = dR[1][1][1] = dR[2][2][2] = 1; break;
    case PSCFG_HEXAGONAL3D:
        ncp = 2; R[0][0] = cp[0]; R[1][0] = -0.5 * cp[0]; R[1][1] = cp[0] * s75; R[2][2] = cp[1];
        dR[0][0][0] = 1; dR[1][0][0] = -0.5; dR[1][1][0] = s75; dR[2][2][1] = 1; break;
    case PSCFG_MONOCLINIC:
        ncp = 4; R[0][0] = cp[0]; R[1][1] = cp[1]; R[2][0] = cp[2] * cos(cp[3]); R[2][2] = cp[2] * sin(cp[3]);
        dR[0][0][0] = 1; dR[1][1][1] = 1; dR[2][0][2] = cos(cp[3]); dR[2][2][2] = sin(cp[3]);
        dR[2][0][3] = -cp[2] * sin(cp[3]); dR[2][2][3] = cp[2] * cos(cp[3]); break;
    default: return false;
    }
    const double twopi = 2.0 * 3.141592653589793;
    double a[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a[i][j] = (i < dim && j < dim) ? R[i][j] : (i == j ? 1.0 : 0.0);
    double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                 a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    double inv[3][3];
    inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    c = Cell();
    c.dim = dim;
    c.ncp = ncp;
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < dim; j++) c.G[i][j] = twopi * inv[j][i];
    double dG[3][3][PSCFG_MAXCP];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < PSCFG_MAXCP; k++) dG[i][j][k] = 0.0;
    for (int k = 0; k < ncp; k++)
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) {
                double s = 0;
                for (int l = 0; l < dim; l++)
                    for (int m = 0; m < dim; m++) s = s - c.G[i][l] * dR[m][l][k] * c.G[m][j];
                dG[i][j][k] = s / twopi;
            }
    for (int k = 0; k < ncp; k++)
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) {
                double s = 0;
                for (int l = 0; l < dim; l++) s = s + c.G[i][l] * dG[j][l][k] + c.G[j][l] * dG[i][l][k];
                c.dGG[k][i][j] = s;
            }
    return true;
}

inline double g_norm(int dim, const int G[3], const double Gb[3][3])
{
    double v[3] = {0, 0, 0};
    for (int j = 0; j < dim; j++)
        for (int i = 0; i < dim; i++) v[j] += G[i] * Gb[i][j];
    double s = 0;
    for (int j = 0; j < dim; j++) s += v[j] * v[j];
    return s;
}

// G_to_bz (src/grid_mod.f90:225-283): images tried +1, 0, -1 per used
// dimension; a later image wins only if smaller by more than 1e-8.
inline void g_to_bz(int dim, const int n[3], const double Gb[3][3], const int G[3], int out[3])
{
    int Gmin[3] = {0, 0, 0}, Gt[3] = {0, 0, 0};
    double gmin = 1.0e10;
    int hi[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) hi[d] = 1;
    for (int i1 = hi[0]; i1 >= -hi[0]; i1--) {
        Gt[0] = G[0] + i1 * n[0];
        for (int i2 = hi[1]; i2 >= -hi[1]; i2--) {
            Gt[1] = (dim > 1) ? G[1] + i2 * n[1] : 0;
            for (int i3 = hi[2]; i3 >= -hi[2]; i3--) {
                Gt[2] = (dim > 2) ? G[2] + i3 * n[2] : 0;
                double g = g_norm(dim, Gt, Gb);
                if (g < gmin - 1.0e-8) {
                    for (int d = 0; d < dim; d++) Gmin[d] = Gt[d];
                    gmin = g;
                }
            }
        }
    }
    out[0] = Gmin[0];
    out[1] = Gmin[1];
    out[2] = Gmin[2];
}

// |G + k|^2 on the full grid for a Bloch wave vector k in reciprocal-basis
// units (calc_ksqgrid_new, src/response_mod.f90:1203-1238): every grid index
// shifted by k is folded by Greal_to_bz (src/grid_mod.f90:286-345, images
// +1, 0, -1 per used dimension, a later image wins only if shorter by more
// than 1e-8); components beyond dim are dropped and ktrans_sq is added.
inline void ksq_bloch(int dim, const int n[3], const double Gb[3][3], const double kvec[3], double ktrans_sq,
                      std::vector<double> &out)
{
    out.assign((size_t)n[0] * n[1] * n[2], 0.0);
    int hi[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) hi[d] = 1;
    for (int i3 = 0; i3 < n[2]; i3++)
        for (int i2 = 0; i2 < n[1]; i2++)
            for (int i1 = 0; i1 < n[0]; i1++) {
                const double g[3] = {i1 + kvec[0], i2 + kvec[1], i3 + kvec[2]};
                double best = 1.0e10;
                for (int s1 = hi[0]; s1 >= -hi[0]; s1--)
                    for (int s2 = hi[1]; s2 >= -hi[1]; s2--)
                        for (int s3 = hi[2]; s3 >= -hi[2]; s3--) {
                            const double t[3] = {g[0] + s1 * n[0], g[1] + s2 * n[1], g[2] + s3 * n[2]};
                            double v[3] = {0, 0, 0};
                            for (int j = 0; j < dim; j++)
                                for (int i = 0; i < dim; i++) v[j] += t[i] * Gb[i][j];
                            double q = 0;
                            for (int j = 0; j < dim; j++) q += v[j] * v[j];
                            if (q < best - 1.0e-8) best = q;
                        }
                out[i1 + (size_t)n[0] * (i2 + (size_t)n[1] * i3)] = best + ktrans_sq;
            }
}

// k^2 on the half grid (make_ksq, src/grid_mod.f90:141-160) and the stress
// weights w(k) * Gbz^T dGG_b Gbz (make_dGsq, src/basis_mod.f90:1993-2014),
// w = 1 on the kx = 0 and kx = n1/2 planes, 2 elsewhere (each interior half
// spectrum entry stands for itself and its conjugate).
inline void make_ksq_dgsq(int dim, const int n[3], const Cell &c, std::vector<double> &ksq, std::vector<double> &wdgsq)
{
    const int n1h = n[0] / 2 + 1;
    const long nk = (long)n1h * n[1] * n[2];
    ksq.assign(nk, 0.0);
    wdgsq.assign((size_t)PSCFG_MAXCP * nk, 0.0);
    for (int i3 = 0; i3 < n[2]; i3++)
        for (int i2 = 0; i2 < n[1]; i2++)
            for (int i1 = 0; i1 < n1h; i1++) {
                int G[3] = {i1, i2, i3}, Gz[3];
                g_to_bz(dim, n, c.G, G, Gz);
                long idx = i1 + (long)n1h * (i2 + (long)n[1] * i3);
                ksq[idx] = g_norm(dim, Gz, c.G);
                double w = (i1 == 0 || (n[0] % 2 == 0 && i1 == n[0] / 2)) ? 1.0 : 2.0;
                for (int b = 0; b < c.ncp; b++) {
                    double v = 0;
                    for (int j = 0; j < dim; j++)
                        for (int l = 0; l < dim; l++) v += (double)Gz[j] * (double)Gz[l] * c.dGG[b][j][l];
                    wdgsq[(size_t)b * nk + idx] = w * v;
                }
            }
}

// Radix plan for a line of length n (radices 8, 4, 2, 3, 5, 7).  Returns
// false if n has another prime factor.
inline bool plan_radices(int n, int *rad, int &nst)
{
    nst = 0;
    int m = n;
    while (m > 1) {
        if (m % 8 == 0 && m != 16) { rad[nst++] = 8; m /= 8; }
        else if (m % 4 == 0) { rad[nst++] = 4; m /= 4; }
        else if (m % 2 == 0) { rad[nst++] = 2; m /= 2; }
        else if (m % 3 == 0) { rad[nst++] = 3; m /= 3; }
        else if (m % 5 == 0) { rad[nst++] = 5; m /= 5; }
        else if (m % 7 == 0) { rad[nst++] = 7; m /= 7; }
        else return false;
        if (nst >= 10) return false;
    }
    return true;
}

}  // namespace pscfg
