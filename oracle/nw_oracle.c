/*
 * nw_oracle.c -- TEST INFRASTRUCTURE ONLY: plain-C restatement of NekWave's
 * single-rank DG-SEM Maxwell right-hand side and LSRK45 time step.
 *
 * This file is the oracle the CUDA path is checked against.  Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it; the
 * product (libnwb) never links, calls or falls back to it.
 *
 * Every routine restates one reference routine with the same floating-point
 * operation order, so that compiled with the same flags (no FMA contraction,
 * see oracle/Makefile) it reproduces the reference's host-compiled kernels bit
 * for bit.  The pin is checked by tests/test_oracle_pin.py against the
 * reference built from its own sources (oracle/_ref) and against the golden
 * vectors in tests/golden/.
 *
 * Reference citations are paths inside the NekWave source tree.
 */
#include "nw_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NWO_PI 3.14159265358979323846

/* Legendre polynomial by Bonnet's recurrence (src/mesh.cpp:19-31). */
static double legendre(int n, double x) {
    if (n == 0) return 1.0;
    if (n == 1) return x;
    double p0 = 1.0, p1 = x, p2 = 0.0;
    for (int k = 1; k < n; ++k) {
        p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
        p0 = p1;
        p1 = p2;
    }
    return p2;
}

/* Derivative of the Legendre polynomial (src/mesh.cpp:35-39). */
static double legendre_deriv(int n, double x) {
    if (n == 0) return 0.0;
    if (n == 1) return 1.0;
    return (n / (x * x - 1.0)) * (x * legendre(n, x) - legendre(n - 1, x));
}

/* Mesh::setupGLL (src/mesh.cpp:64-145). */
void nwo_gll(int N, double* z, double* w, double* D, double* w3) {
    int p = N - 1;
    for (int i = 0; i < N * N; ++i) D[i] = 0.0;
    if (N == 1) {
        z[0] = 0.0;
        w[0] = 2.0;
        D[0] = 0.0;
    } else {
        z[0] = -1.0;
        z[N - 1] = 1.0;
        /* Newton on L'_p with a Chebyshev start (src/mesh.cpp:84-98) */
        for (int i = 1; i < N - 1; ++i) {
            double xi = -cos((NWO_PI * i) / p);
            for (int it = 0; it < 20; ++it) {
                double L = legendre(p, xi);
                double Ld = legendre_deriv(p, xi);
                double Ldd = (2.0 * xi * Ld - p * (p + 1.0) * L) / (1.0 - xi * xi);
                double delta = Ld / Ldd;
                xi -= delta;
                if (fabs(delta) < 1e-15) break;
            }
            z[i] = xi;
        }
        /* w_i = 2 / (p (p+1) L_p(x_i)^2) (src/mesh.cpp:101-104) */
        for (int i = 0; i < N; ++i) {
            double L = legendre(p, z[i]);
            w[i] = 2.0 / (p * (p + 1.0) * L * L);
        }
        /* D_ij = L_p(x_i) / (L_p(x_j) (x_i - x_j)), corners -+p(p+1)/4
         * (src/mesh.cpp:113-131) */
        double d0 = p * (p + 1.0) / 4.0;
        for (int i = 0; i < N; ++i) {
            for (int j = 0; j < N; ++j) {
                int idx = i + j * N;
                if (i != j) {
                    double Li = legendre(p, z[i]);
                    double Lj = legendre(p, z[j]);
                    D[idx] = Li / (Lj * (z[i] - z[j]));
                } else if (i == 0 && j == 0) {
                    D[idx] = -d0;
                } else if (i == p && j == p) {
                    D[idx] = d0;
                } else {
                    D[idx] = 0.0;
                }
            }
        }
    }
    /* w3_ijk = w_i w_j w_k (src/mesh.cpp:137-144) */
    if (w3) {
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i)
                    w3[i + N * (j + N * k)] = w[i] * w[j] * w[k];
    }
}

/* Mesh::getFaceNodeVolIndex (src/mesh.cpp:955-981). */
static int face_node(int N, int e, int f, int p, int q) {
    int i = 0, j = 0, k = 0;
    switch (f) {
        case 0: i = p; j = 0; k = q; break;
        case 1: i = N - 1; j = p; k = q; break;
        case 2: i = p; j = N - 1; k = q; break;
        case 3: i = 0; j = p; k = q; break;
        case 4: i = p; j = q; k = 0; break;
        case 5: i = p; j = q; k = N - 1; break;
        default: break;
    }
    return e * N * N * N + i + N * (j + N * k);
}

/* Face kinds of createBoxMesh (src/mesh.cpp:718-826). */
enum { FACE_E = 0, FACE_PERIODIC = 1, FACE_PEC = 2 };

/* One element's trilinear geometry (src/mesh.cpp:188-314). */
static void element_metrics(int N, const double* zg, const double c[8][3], int off,
                            double* x, double* y, double* z, double* jac, double* met,
                            long npts) {
    for (int k = 0; k < N; ++k) {
        double t = zg[k];
        for (int j = 0; j < N; ++j) {
            double s = zg[j];
            for (int i = 0; i < N; ++i) {
                double r = zg[i];
                long pt = off + i + N * (j + N * k);
                double Nf[8], dr[8], ds[8], dt[8];
                Nf[0] = 0.125 * (1.0 - r) * (1.0 - s) * (1.0 - t);
                Nf[1] = 0.125 * (1.0 + r) * (1.0 - s) * (1.0 - t);
                Nf[2] = 0.125 * (1.0 + r) * (1.0 + s) * (1.0 - t);
                Nf[3] = 0.125 * (1.0 - r) * (1.0 + s) * (1.0 - t);
                Nf[4] = 0.125 * (1.0 - r) * (1.0 - s) * (1.0 + t);
                Nf[5] = 0.125 * (1.0 + r) * (1.0 - s) * (1.0 + t);
                Nf[6] = 0.125 * (1.0 + r) * (1.0 + s) * (1.0 + t);
                Nf[7] = 0.125 * (1.0 - r) * (1.0 + s) * (1.0 + t);

                dr[0] = -0.125 * (1.0 - s) * (1.0 - t);
                dr[1] =  0.125 * (1.0 - s) * (1.0 - t);
                dr[2] =  0.125 * (1.0 + s) * (1.0 - t);
                dr[3] = -0.125 * (1.0 + s) * (1.0 - t);
                dr[4] = -0.125 * (1.0 - s) * (1.0 + t);
                dr[5] =  0.125 * (1.0 - s) * (1.0 + t);
                dr[6] =  0.125 * (1.0 + s) * (1.0 + t);
                dr[7] = -0.125 * (1.0 + s) * (1.0 + t);

                ds[0] = -0.125 * (1.0 - r) * (1.0 - t);
                ds[1] = -0.125 * (1.0 + r) * (1.0 - t);
                ds[2] =  0.125 * (1.0 + r) * (1.0 - t);
                ds[3] =  0.125 * (1.0 - r) * (1.0 - t);
                ds[4] = -0.125 * (1.0 - r) * (1.0 + t);
                ds[5] = -0.125 * (1.0 + r) * (1.0 + t);
                ds[6] =  0.125 * (1.0 + r) * (1.0 + t);
                ds[7] =  0.125 * (1.0 - r) * (1.0 + t);

                dt[0] = -0.125 * (1.0 - r) * (1.0 - s);
                dt[1] = -0.125 * (1.0 + r) * (1.0 - s);
                dt[2] = -0.125 * (1.0 + r) * (1.0 + s);
                dt[3] = -0.125 * (1.0 - r) * (1.0 + s);
                dt[4] =  0.125 * (1.0 - r) * (1.0 - s);
                dt[5] =  0.125 * (1.0 + r) * (1.0 - s);
                dt[6] =  0.125 * (1.0 + r) * (1.0 + s);
                dt[7] =  0.125 * (1.0 - r) * (1.0 + s);

                double px = 0.0, py = 0.0, pz = 0.0;
                double xr = 0.0, yr = 0.0, zr = 0.0;
                double xs = 0.0, ys = 0.0, zs = 0.0;
                double xt = 0.0, yt = 0.0, zt = 0.0;
                for (int a = 0; a < 8; ++a) {
                    double vx = c[a][0], vy = c[a][1], vz = c[a][2];
                    px += Nf[a] * vx;
                    py += Nf[a] * vy;
                    pz += Nf[a] * vz;
                    xr += dr[a] * vx;
                    yr += dr[a] * vy;
                    zr += dr[a] * vz;
                    xs += ds[a] * vx;
                    ys += ds[a] * vy;
                    zs += ds[a] * vz;
                    xt += dt[a] * vx;
                    yt += dt[a] * vy;
                    zt += dt[a] * vz;
                }
                x[pt] = px;
                y[pt] = py;
                z[pt] = pz;
                double detJ = xr * (ys * zt - yt * zs)
                            - xs * (yr * zt - yt * zr)
                            + xt * (yr * zs - ys * zr);
                jac[pt] = detJ;
                double invJ = 1.0 / detJ;
                met[0 * npts + pt] = invJ * (ys * zt - yt * zs);  /* rx */
                met[1 * npts + pt] = invJ * (yt * zr - yr * zt);  /* sx */
                met[2 * npts + pt] = invJ * (yr * zs - ys * zr);  /* tx */
                met[3 * npts + pt] = invJ * (xt * zs - xs * zt);  /* ry */
                met[4 * npts + pt] = invJ * (xr * zt - xt * zr);  /* sy */
                met[5 * npts + pt] = invJ * (xs * zr - xr * zs);  /* ty */
                met[6 * npts + pt] = invJ * (xs * yt - xt * ys);  /* rz */
                met[7 * npts + pt] = invJ * (xt * yr - xr * yt);  /* sz */
                met[8 * npts + pt] = invJ * (xr * ys - xs * yr);  /* tz */
            }
        }
    }
}

int nwo_hex_mesh(int N, int nelt, const double* corners, const int* fkind,
                 const int* fnb, const int* fnf,
                 double* x, double* y, double* z, double* jac, double* met,
                 int* vmin, int* vplus, int* bc,
                 double* nx, double* ny, double* nz, double* dA) {
    if (N < 2 || N > 16 || nelt < 1) return -1;
    int N3 = N * N * N;
    long npts = (long)nelt * N3;
    double zg[16], wg[16], D[256];
    nwo_gll(N, zg, wg, D, NULL);
    for (int e = 0; e < nelt; ++e) {
        double c[8][3];
        for (int a = 0; a < 8; ++a)
            for (int d = 0; d < 3; ++d) c[a][d] = corners[((long)e * 8 + a) * 3 + d];
        element_metrics(N, zg, c, e * N3, x, y, z, jac, met, npts);
    }

    /* Mesh::setupFaceData (src/mesh.cpp:985-1080) + flattening
     * (src/dg_solver.cpp:76-112), face points in (element, face, q, p) order. */
    const double* rxa = met + 0 * npts; const double* sxa = met + 1 * npts;
    const double* txa = met + 2 * npts; const double* rya = met + 3 * npts;
    const double* sya = met + 4 * npts; const double* tya = met + 5 * npts;
    const double* rza = met + 6 * npts; const double* sza = met + 7 * npts;
    const double* tza = met + 8 * npts;
    int NN = N * N;
#pragma omp parallel for schedule(static)
    for (int ef = 0; ef < 6 * nelt; ++ef) {
        int eA = ef / 6, fA = ef % 6;
        int kind = fkind[ef], eB = fnb[ef], fB = fnf[ef];
        for (int qA = 0; qA < N; ++qA) {
            for (int pA = 0; pA < N; ++pA) {
                long fp = (long)ef * NN + qA * N + pA;
                int vM = face_node(N, eA, fA, pA, qA);
                double J = jac[vM];
                double w2 = wg[pA] * wg[qA];
                double Nx = 0.0, Ny = 0.0, Nz = 0.0;
                switch (fA) {
                    case 0: Nx = -J * sxa[vM]; Ny = -J * sya[vM]; Nz = -J * sza[vM]; break;
                    case 1: Nx = +J * rxa[vM]; Ny = +J * rya[vM]; Nz = +J * rza[vM]; break;
                    case 2: Nx = +J * sxa[vM]; Ny = +J * sya[vM]; Nz = +J * sza[vM]; break;
                    case 3: Nx = -J * rxa[vM]; Ny = -J * rya[vM]; Nz = -J * rza[vM]; break;
                    case 4: Nx = -J * txa[vM]; Ny = -J * tya[vM]; Nz = -J * tza[vM]; break;
                    case 5: Nx = +J * txa[vM]; Ny = +J * tya[vM]; Nz = +J * tza[vM]; break;
                }
                double L = sqrt(Nx * Nx + Ny * Ny + Nz * Nz);
                nx[fp] = (L > 1e-14) ? (Nx / L) : 0.0;
                ny[fp] = (L > 1e-14) ? (Ny / L) : 0.0;
                nz[fp] = (L > 1e-14) ? (Nz / L) : 0.0;
                dA[fp] = L * w2;
                vmin[fp] = vM;
                int vP;
                if (kind == FACE_PEC || eB < 0) {
                    vP = -1;
                } else if (kind == FACE_PERIODIC) {
                    vP = face_node(N, eB, fB, pA, qA);
                } else {
                    /* coordinate match within 1e-10 (src/mesh.cpp:1049-1069) */
                    double xA = x[vM], yA = y[vM], zA = z[vM];
                    vP = -1;
                    for (int qB = 0; qB < N && vP < 0; ++qB) {
                        for (int pB = 0; pB < N; ++pB) {
                            int vB = face_node(N, eB, fB, pB, qB);
                            double ddx = xA - x[vB];
                            double ddy = yA - y[vB];
                            double ddz = zA - z[vB];
                            if (ddx * ddx + ddy * ddy + ddz * ddz < 1e-10) { vP = vB; break; }
                        }
                    }
                }
                vplus[fp] = vP;
                /* bcCode: PEC -> 1, "E"/"PERIODIC" -> 0; no neighbour forces 1
                 * (src/dg_solver.cpp:92-104) */
                int code = (kind == FACE_PEC) ? 1 : 0;
                if (vP < 0 && code == 0) code = 1;
                bc[fp] = code;
            }
        }
    }
    return 0;
}

int nwo_box_corners(int nelx, int nely, int nelz,
                    double xmin, double xmax, double ymin, double ymax,
                    double zmin, double zmax, int px, int py, int pz,
                    double* corners, int* fkind, int* fnb, int* fnf) {
    if (nelx < 1 || nely < 1 || nelz < 1) return -1;
    double dx = (xmax - xmin) / nelx;
    double dy = (ymax - ymin) / nely;
    double dz = (zmax - zmin) / nelz;
#define EIDX(a, b, c) ((a) + nelx * ((b) + nely * (c)))
    for (int ez = 0; ez < nelz; ++ez) {
        double z0 = zmin + ez * dz, z1 = z0 + dz;
        for (int ey = 0; ey < nely; ++ey) {
            double y0 = ymin + ey * dy, y1 = y0 + dy;
            for (int ex = 0; ex < nelx; ++ex) {
                double x0 = xmin + ex * dx, x1 = x0 + dx;
                int e = EIDX(ex, ey, ez);
                double c[8][3] = {{x0, y0, z0}, {x1, y0, z0}, {x1, y1, z0}, {x0, y1, z0},
                                  {x0, y0, z1}, {x1, y0, z1}, {x1, y1, z1}, {x0, y1, z1}};
                for (int a = 0; a < 8; ++a)
                    for (int d = 0; d < 3; ++d) corners[((long)e * 8 + a) * 3 + d] = c[a][d];
                int* K = fkind + 6 * e;
                int* B = fnb + 6 * e;
                int* F = fnf + 6 * e;
                /* face 0: s=-1 */
                if (ey > 0) { K[0] = FACE_E; B[0] = EIDX(ex, ey - 1, ez); F[0] = 2; }
                else if (py) { K[0] = FACE_PERIODIC; B[0] = EIDX(ex, nely - 1, ez); F[0] = 2; }
                else { K[0] = FACE_PEC; B[0] = -1; F[0] = -1; }
                /* face 1: r=+1 */
                if (ex < nelx - 1) { K[1] = FACE_E; B[1] = EIDX(ex + 1, ey, ez); F[1] = 3; }
                else if (px) { K[1] = FACE_PERIODIC; B[1] = EIDX(0, ey, ez); F[1] = 3; }
                else { K[1] = FACE_PEC; B[1] = -1; F[1] = -1; }
                /* face 2: s=+1 */
                if (ey < nely - 1) { K[2] = FACE_E; B[2] = EIDX(ex, ey + 1, ez); F[2] = 0; }
                else if (py) { K[2] = FACE_PERIODIC; B[2] = EIDX(ex, 0, ez); F[2] = 0; }
                else { K[2] = FACE_PEC; B[2] = -1; F[2] = -1; }
                /* face 3: r=-1 */
                if (ex > 0) { K[3] = FACE_E; B[3] = EIDX(ex - 1, ey, ez); F[3] = 1; }
                else if (px) { K[3] = FACE_PERIODIC; B[3] = EIDX(nelx - 1, ey, ez); F[3] = 1; }
                else { K[3] = FACE_PEC; B[3] = -1; F[3] = -1; }
                /* face 4: t=-1 */
                if (ez > 0) { K[4] = FACE_E; B[4] = EIDX(ex, ey, ez - 1); F[4] = 5; }
                else if (pz) { K[4] = FACE_PERIODIC; B[4] = EIDX(ex, ey, nelz - 1); F[4] = 5; }
                else { K[4] = FACE_PEC; B[4] = -1; F[4] = -1; }
                /* face 5: t=+1 */
                if (ez < nelz - 1) { K[5] = FACE_E; B[5] = EIDX(ex, ey, ez + 1); F[5] = 4; }
                else if (pz) { K[5] = FACE_PERIODIC; B[5] = EIDX(ex, ey, 0); F[5] = 4; }
                else { K[5] = FACE_PEC; B[5] = -1; F[5] = -1; }
            }
        }
    }
#undef EIDX
    return 0;
}

int nwo_box_mesh(int N, int nelx, int nely, int nelz,
                 double xmin, double xmax, double ymin, double ymax,
                 double zmin, double zmax, int px, int py, int pz,
                 double* x, double* y, double* z, double* jac, double* met,
                 int* vmin, int* vplus, int* bc,
                 double* nx, double* ny, double* nz, double* dA) {
    if (N < 2 || N > 16 || nelx < 1 || nely < 1 || nelz < 1) return -1;
    int nelt = nelx * nely * nelz;
    double* corners = (double*)malloc(sizeof(double) * 24 * (size_t)nelt);
    int* fkind = (int*)malloc(sizeof(int) * 6 * (size_t)nelt);
    int* fnb = (int*)malloc(sizeof(int) * 6 * (size_t)nelt);
    int* fnf = (int*)malloc(sizeof(int) * 6 * (size_t)nelt);
    int rc = -1;
    if (corners && fkind && fnb && fnf) {
        nwo_box_corners(nelx, nely, nelz, xmin, xmax, ymin, ymax, zmin, zmax, px, py, pz,
                        corners, fkind, fnb, fnf);
        rc = nwo_hex_mesh(N, nelt, corners, fkind, fnb, fnf, x, y, z, jac, met, vmin, vplus,
                          bc, nx, ny, nz, dA);
    }
    free(corners); free(fkind); free(fnb); free(fnf);
    return rc;
}

/* Mesh::computeMinNodeDistance (src/mesh.cpp:883-930). */
double nwo_dxmin(int N, int nelt, const double* x, const double* y, const double* z) {
    double minD2 = 1.0e20;
    int N3 = N * N * N;
    for (int e = 0; e < nelt; ++e) {
        long off = (long)e * N3;
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i) {
                    long idx = off + i + N * (j + N * k);
                    double x0 = x[idx], y0 = y[idx], z0 = z[idx];
                    long nb[3] = {i + 1 < N ? off + (i + 1) + N * (j + N * k) : -1,
                                  j + 1 < N ? off + i + N * ((j + 1) + N * k) : -1,
                                  k + 1 < N ? off + i + N * (j + N * (k + 1)) : -1};
                    for (int d = 0; d < 3; ++d) {
                        if (nb[d] < 0) continue;
                        double dx = x[nb[d]] - x0, dy = y[nb[d]] - y0, dz = z[nb[d]] - z0;
                        double d2 = dx * dx + dy * dy + dz * dz;
                        if (d2 < minD2) minD2 = d2;
                    }
                }
    }
    return sqrt(minD2);
}

/* gpu_volume_curl_kernel (src/device/dg_kernels.cu:41-155) for one element,
 * input components u1..u3, output w1..w3 scaled by sign. */
static void volume_curl_elem(int N, int e, const double* D, const double* w3g,
                             const double* jac, const double* met, long npts,
                             const double* u1, const double* u2, const double* u3,
                             double* o1, double* o2, double* o3, double sign) {
    int N2 = N * N, N3 = N2 * N;
    long base = (long)e * N3;
    const double* s1 = u1 + base;
    const double* s2 = u2 + base;
    const double* s3 = u3 + base;
    for (int m = 0; m < N3; ++m) {
        long p = base + m;
        int i = m % N, j = (m / N) % N, k = m / N2;
        double u1r = 0.0, u1s = 0.0, u1t = 0.0;
        double u2r = 0.0, u2s = 0.0, u2t = 0.0;
        double u3r = 0.0, u3s = 0.0, u3t = 0.0;
        for (int l = 0; l < N; ++l) {
            double d_il = D[i + l * N];
            double d_jl = D[j + l * N];
            double d_kl = D[k + l * N];
            int ir = l + j * N + k * N2;
            u1r += d_il * s1[ir];
            u2r += d_il * s2[ir];
            u3r += d_il * s3[ir];
            int is = i + l * N + k * N2;
            u1s += d_jl * s1[is];
            u2s += d_jl * s2[is];
            u3s += d_jl * s3[is];
            int it = i + j * N + l * N2;
            u1t += d_kl * s1[it];
            u2t += d_kl * s2[it];
            u3t += d_kl * s3[it];
        }
        double w = w3g[m] * jac[p];
        double u1rw = u1r * w, u1sw = u1s * w, u1tw = u1t * w;
        double u2rw = u2r * w, u2sw = u2s * w, u2tw = u2t * w;
        double u3rw = u3r * w, u3sw = u3s * w, u3tw = u3t * w;
        double rx = met[0 * npts + p], sx = met[1 * npts + p], tx = met[2 * npts + p];
        double ry = met[3 * npts + p], sy = met[4 * npts + p], ty = met[5 * npts + p];
        double rz = met[6 * npts + p], sz = met[7 * npts + p], tz = met[8 * npts + p];
        double c1 = (u3rw * ry + u3sw * sy + u3tw * ty) - (u2rw * rz + u2sw * sz + u2tw * tz);
        double c2 = (u1rw * rz + u1sw * sz + u1tw * tz) - (u3rw * rx + u3sw * sx + u3tw * tx);
        double c3 = (u2rw * rx + u2sw * sx + u2tw * tx) - (u1rw * ry + u1sw * sy + u1tw * ty);
        o1[p] = sign * c1;
        o2[p] = sign * c2;
        o3[p] = sign * c3;
    }
}

/* Off: the reference's behaviour (every bc != 0 point is a PEC mirror).  On: bc 2
   points are PMC mirrors, the checker of libnwb's NWB_SOLVER_TRUE_PMC option. */
static int g_true_pmc = 0;
void nwo_set_true_pmc(int on) { g_true_pmc = on != 0; }

void nwo_rhs(int N, int nelt, const double* D, const double* w3,
             const double* jac, const double* met,
             int nfp, const int* vmin, const int* vplus, const int* bc,
             const double* nx, const double* ny, const double* nz, const double* dA,
             double c0, const double* u, double* rhs) {
    long N3 = (long)N * N * N;
    long npts = (long)nelt * N3;
    const double* Ex = u + 0 * npts; const double* Ey = u + 1 * npts;
    const double* Ez = u + 2 * npts; const double* Hx = u + 3 * npts;
    const double* Hy = u + 4 * npts; const double* Hz = u + 5 * npts;

    /* +curl H -> resE, -curl E -> resH (src/dg_solver.cpp:393-413) */
#pragma omp parallel for schedule(static)
    for (int e = 0; e < nelt; ++e) {
        volume_curl_elem(N, e, D, w3, jac, met, npts, Hx, Hy, Hz,
                         rhs + 0 * npts, rhs + 1 * npts, rhs + 2 * npts, 1.0);
        volume_curl_elem(N, e, D, w3, jac, met, npts, Ex, Ey, Ez,
                         rhs + 3 * npts, rhs + 4 * npts, rhs + 5 * npts, -1.0);
    }

    /* restrict + flux (src/device/dg_kernels.cu:170-304) */
    double* flux = (double*)malloc(sizeof(double) * 6 * (size_t)nfp);
    if (!flux) abort();
#pragma omp parallel for schedule(static)
    for (int p = 0; p < nfp; ++p) {
        int vM = vmin[p];
        double Ex_m = u[0 * npts + vM], Ey_m = u[1 * npts + vM], Ez_m = u[2 * npts + vM];
        double Hx_m = u[3 * npts + vM], Hy_m = u[4 * npts + vM], Hz_m = u[5 * npts + vM];
        double dEx, dEy, dEz, dHx, dHy, dHz;
        if (g_true_pmc && bc[p] == 2) {
            /* option, not in the reference (which mirrors PMC faces as PEC):
               PMC mirror [[E]] = 0, [[H]] = -2 H^- */
            dEx = 0.0; dEy = 0.0; dEz = 0.0;
            dHx = -2.0 * Hx_m; dHy = -2.0 * Hy_m; dHz = -2.0 * Hz_m;
        } else if (bc[p] || vplus[p] < 0) {
            dEx = -2.0 * Ex_m; dEy = -2.0 * Ey_m; dEz = -2.0 * Ez_m;
            dHx = 0.0; dHy = 0.0; dHz = 0.0;
        } else {
            long vP = vplus[p];
            dEx = u[0 * npts + vP] - Ex_m;
            dEy = u[1 * npts + vP] - Ey_m;
            dEz = u[2 * npts + vP] - Ez_m;
            dHx = u[3 * npts + vP] - Hx_m;
            dHy = u[4 * npts + vP] - Hy_m;
            dHz = u[5 * npts + vP] - Hz_m;
        }
        double n_x = nx[p], n_y = ny[p], n_z = nz[p];
        double nxE_x = n_y * dEz - n_z * dEy;
        double nxE_y = n_z * dEx - n_x * dEz;
        double nxE_z = n_x * dEy - n_y * dEx;
        double nxH_x = n_y * dHz - n_z * dHy;
        double nxH_y = n_z * dHx - n_x * dHz;
        double nxH_z = n_x * dHy - n_y * dHx;
        double nxnxE_x = n_y * nxE_z - n_z * nxE_y;
        double nxnxE_y = n_z * nxE_x - n_x * nxE_z;
        double nxnxE_z = n_x * nxE_y - n_y * nxE_x;
        double nxnxH_x = n_y * nxH_z - n_z * nxH_y;
        double nxnxH_y = n_z * nxH_x - n_x * nxH_z;
        double nxnxH_z = n_x * nxH_y - n_y * nxH_x;
        flux[0 * (size_t)nfp + p] = -0.5 * nxE_x - 0.5 * c0 * nxnxH_x;
        flux[1 * (size_t)nfp + p] = -0.5 * nxE_y - 0.5 * c0 * nxnxH_y;
        flux[2 * (size_t)nfp + p] = -0.5 * nxE_z - 0.5 * c0 * nxnxH_z;
        flux[3 * (size_t)nfp + p] = +0.5 * nxH_x - 0.5 * c0 * nxnxE_x;
        flux[4 * (size_t)nfp + p] = +0.5 * nxH_y - 0.5 * c0 * nxnxE_y;
        flux[5 * (size_t)nfp + p] = +0.5 * nxH_z - 0.5 * c0 * nxnxE_z;
    }

    /* lift (src/device/dg_kernels.cu:316-338), summed in face-point order so the
     * oracle is deterministic; the reference's atomics may sum in any order. */
    for (int p = 0; p < nfp; ++p) {
        long vM = vmin[p];
        double a = dA[p];
        rhs[0 * npts + vM] += a * flux[3 * (size_t)nfp + p];
        rhs[1 * npts + vM] += a * flux[4 * (size_t)nfp + p];
        rhs[2 * npts + vM] += a * flux[5 * (size_t)nfp + p];
        rhs[3 * npts + vM] += a * flux[0 * (size_t)nfp + p];
        rhs[4 * npts + vM] += a * flux[1 * (size_t)nfp + p];
        rhs[5 * npts + vM] += a * flux[2 * (size_t)nfp + p];
    }
    free(flux);

    /* inverse mass, eps = mu = 1 (src/device/dg_kernels.cu:353-382) */
#pragma omp parallel for schedule(static)
    for (long kk = 0; kk < npts; ++kk) {
        long i = kk % N3;
        const double eps = 1.0, mu = 1.0;
        double invE = 1.0 / (eps * jac[kk] * w3[i]);
        double invH = 1.0 / (mu * jac[kk] * w3[i]);
        rhs[0 * npts + kk] *= invE;
        rhs[1 * npts + kk] *= invE;
        rhs[2 * npts + kk] *= invE;
        rhs[3 * npts + kk] *= invH;
        rhs[4 * npts + kk] *= invH;
        rhs[5 * npts + kk] *= invH;
    }
}

/* Carpenter-Kennedy LSRK45 (src/dg_solver.cpp:58-69). */
void nwo_lsrk45(double* a5, double* b5) {
    a5[0] = 0.0;
    a5[1] = -567301805773.0 / 1357537059087.0;
    a5[2] = -2404267990393.0 / 2016746695238.0;
    a5[3] = -3550918686646.0 / 2091501179385.0;
    a5[4] = -1275806237668.0 / 842570457699.0;
    b5[0] = 1432997174477.0 / 9575080441755.0;
    b5[1] = 5161836677717.0 / 13612068292357.0;
    b5[2] = 1720146321549.0 / 2090206949498.0;
    b5[3] = 3134564353537.0 / 4481467310338.0;
    b5[4] = 2277821191437.0 / 14882151754819.0;
}

void nwo_step(int N, int nelt, const double* D, const double* w3,
              const double* jac, const double* met,
              int nfp, const int* vmin, const int* vplus, const int* bc,
              const double* nx, const double* ny, const double* nz, const double* dA,
              double c0, double dt, int nsteps, double* u, double* k) {
    long npts = (long)nelt * N * N * N;
    long ntot = 6 * npts;
    double a5[5], b5[5];
    nwo_lsrk45(a5, b5);
    double* rhs = (double*)malloc(sizeof(double) * (size_t)ntot);
    if (!rhs) abort();
    for (int s = 0; s < nsteps; ++s) {
        for (int st = 0; st < 5; ++st) {
            nwo_rhs(N, nelt, D, w3, jac, met, nfp, vmin, vplus, bc, nx, ny, nz, dA,
                    c0, u, rhs);
            double as = a5[st], bs = b5[st];
            /* gpu_lsrk45_update_kernel (src/device/dg_kernels.cu:393-408) */
#pragma omp parallel for schedule(static)
            for (long i = 0; i < ntot; ++i) {
                double ki = as * k[i] + dt * rhs[i];
                k[i] = ki;
                u[i] += bs * ki;
            }
        }
    }
    free(rhs);
}

double nwo_energy(int N, int nelt, const double* w, const double* J, const double* u) {
    long Np = (long)N * N * N;
    long npts = (long)nelt * Np;
    const double* Ex = u + 0 * npts; const double* Ey = u + 1 * npts;
    const double* Ez = u + 2 * npts; const double* Hx = u + 3 * npts;
    const double* Hy = u + 4 * npts; const double* Hz = u + 5 * npts;
    double energy = 0.0;
    for (int e = 0; e < nelt; ++e)
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i) {
                    long p = e * Np + k * N * N + j * N + i;
                    double dV = J[p] * w[i] * w[j] * w[k];
                    double eSq = Ex[p] * Ex[p] + Ey[p] * Ey[p] + Ez[p] * Ez[p];
                    double hSq = Hx[p] * Hx[p] + Hy[p] * Hy[p] + Hz[p] * Hz[p];
                    energy += 0.5 * (eSq + hSq) * dV;
                }
    return energy;
}

int nwo_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
