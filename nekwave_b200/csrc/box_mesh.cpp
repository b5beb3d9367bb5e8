// box_mesh.cpp -- structured box mesh with the arrays the hot path consumes.
//
// Replaces Mesh::createBoxMesh (src/mesh.cpp:683-843) for callers of libnwb that
// do not link the reference's Mesh.  Geometry uses the reference's trilinear
// map and its operation order (src/mesh.cpp:188-314), so the node coordinates,
// Jacobians and metrics are the reference's values.  Face data follows
// Mesh::setupFaceData (src/mesh.cpp:985-1080), except that the neighbour node of
// an interior face point is found structurally: on a conforming box mesh the
// point (p,q) of face f meets the point (p,q) of the opposite face of the
// neighbour (the match the reference finds by an O(N^4) coordinate search per
// face, src/mesh.cpp:1049-1069).
#include "nwb.h"
#include "nwb_internal.h"

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

extern "C" void nwb_set_error_(const char* msg);

struct nwb_box_mesh {
    int N = 0, nelt = 0;
    std::vector<double> z, w, D, w3, x, y, zc, jac;
    std::vector<double> met[9];
    std::vector<int> vmin, vplus, bc;
    std::vector<double> nx, ny, nz, dA;
};

namespace {

double legendre(int n, double x) {
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

double legendre_deriv(int n, double x) {
    if (n == 0) return 0.0;
    if (n == 1) return 1.0;
    return (n / (x * x - 1.0)) * (x * legendre(n, x) - legendre(n - 1, x));
}

}  // namespace

namespace nwb {

// GLL nodes, weights and the collocation derivative matrix (column-major
// D[i + j N] = l_j'(x_i)): Newton on L'_p from a Chebyshev start, weights
// 2/(p(p+1)L_p^2), corner entries -+p(p+1)/4 (src/mesh.cpp:64-145).
void gll(int N, std::vector<double>& z, std::vector<double>& w, std::vector<double>& D) {
    const int p = N - 1;
    z.assign(N, 0.0);
    w.assign(N, 0.0);
    D.assign(static_cast<size_t>(N) * N, 0.0);
    z[0] = -1.0;
    z[N - 1] = 1.0;
    for (int i = 1; i < N - 1; ++i) {
        double xi = -std::cos((M_PI * i) / p);
        for (int it = 0; it < 20; ++it) {
            const double L = legendre(p, xi);
            const double Ld = legendre_deriv(p, xi);
            const double Ldd = (2.0 * xi * Ld - p * (p + 1.0) * L) / (1.0 - xi * xi);
            const double delta = Ld / Ldd;
            xi -= delta;
            if (std::abs(delta) < 1e-15) break;
        }
        z[i] = xi;
    }
    for (int i = 0; i < N; ++i) {
        const double L = legendre(p, z[i]);
        w[i] = 2.0 / (p * (p + 1.0) * L * L);
    }
    const double d0 = p * (p + 1.0) / 4.0;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            double v;
            if (i != j) v = legendre(p, z[i]) / (legendre(p, z[j]) * (z[i] - z[j]));
            else if (i == 0) v = -d0;
            else if (i == p) v = d0;
            else v = 0.0;
            D[i + j * N] = v;
        }
}

// z with D z = 1, z[0] = -1: least squares over all N rows for z[1..N-1] (normal
// equations of the N x (N-1) system D[:, 1:] z[1:] = 1 + D[:, 0], rank N-1),
// Gaussian elimination with partial pivoting.
void line_coords(int N, const double* D, double* z) {
    const int n = N - 1;
    double M[9][10] = {};
    for (int a = 0; a < n; ++a) {
        for (int b = 0; b < n; ++b) {
            double s = 0.0;
            for (int i = 0; i < N; ++i) s += D[i + N * (a + 1)] * D[i + N * (b + 1)];
            M[a][b] = s;
        }
        double r = 0.0;
        for (int i = 0; i < N; ++i) r += D[i + N * (a + 1)] * (1.0 + D[i]);
        M[a][n] = r;
    }
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(M[r][c]) > std::abs(M[piv][c])) piv = r;
        for (int x = 0; x <= n; ++x) std::swap(M[c][x], M[piv][x]);
        for (int r = c + 1; r < n; ++r) {
            const double f = M[r][c] / M[c][c];
            for (int x = c; x <= n; ++x) M[r][x] -= f * M[c][x];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        double s = M[c][n];
        for (int x = c + 1; x < n; ++x) s -= M[c][x] * z[x + 1];
        z[c + 1] = s / M[c][c];
    }
    z[0] = -1.0;
}

// Trilinear map of one element with the reference's operation order
// (src/mesh.cpp:188-314): position, J and J^{-T} (rx,sx,tx,ry,sy,ty,rz,sz,tz)
// at reference point (r,s,t).
void trilinear_point(const double c[8][3], double r, double s, double t, double* X, double* J,
                     double met[9]) {
    const double Nf[8] = {
        0.125 * (1.0 - r) * (1.0 - s) * (1.0 - t), 0.125 * (1.0 + r) * (1.0 - s) * (1.0 - t),
        0.125 * (1.0 + r) * (1.0 + s) * (1.0 - t), 0.125 * (1.0 - r) * (1.0 + s) * (1.0 - t),
        0.125 * (1.0 - r) * (1.0 - s) * (1.0 + t), 0.125 * (1.0 + r) * (1.0 - s) * (1.0 + t),
        0.125 * (1.0 + r) * (1.0 + s) * (1.0 + t), 0.125 * (1.0 - r) * (1.0 + s) * (1.0 + t)};
    const double dr[8] = {
        -0.125 * (1.0 - s) * (1.0 - t), 0.125 * (1.0 - s) * (1.0 - t),
        0.125 * (1.0 + s) * (1.0 - t), -0.125 * (1.0 + s) * (1.0 - t),
        -0.125 * (1.0 - s) * (1.0 + t), 0.125 * (1.0 - s) * (1.0 + t),
        0.125 * (1.0 + s) * (1.0 + t), -0.125 * (1.0 + s) * (1.0 + t)};
    const double ds[8] = {
        -0.125 * (1.0 - r) * (1.0 - t), -0.125 * (1.0 + r) * (1.0 - t),
        0.125 * (1.0 + r) * (1.0 - t), 0.125 * (1.0 - r) * (1.0 - t),
        -0.125 * (1.0 - r) * (1.0 + t), -0.125 * (1.0 + r) * (1.0 + t),
        0.125 * (1.0 + r) * (1.0 + t), 0.125 * (1.0 - r) * (1.0 + t)};
    const double dt[8] = {
        -0.125 * (1.0 - r) * (1.0 - s), -0.125 * (1.0 + r) * (1.0 - s),
        -0.125 * (1.0 + r) * (1.0 + s), -0.125 * (1.0 - r) * (1.0 + s),
        0.125 * (1.0 - r) * (1.0 - s), 0.125 * (1.0 + r) * (1.0 - s),
        0.125 * (1.0 + r) * (1.0 + s), 0.125 * (1.0 - r) * (1.0 + s)};
    double px = 0, py = 0, pz = 0, xr = 0, yr = 0, zr = 0, xs = 0, ys = 0, zs = 0, xt = 0, yt = 0, zt = 0;
    for (int a = 0; a < 8; ++a) {
        const double vx = c[a][0], vy = c[a][1], vz = c[a][2];
        px += Nf[a] * vx; py += Nf[a] * vy; pz += Nf[a] * vz;
        xr += dr[a] * vx; yr += dr[a] * vy; zr += dr[a] * vz;
        xs += ds[a] * vx; ys += ds[a] * vy; zs += ds[a] * vz;
        xt += dt[a] * vx; yt += dt[a] * vy; zt += dt[a] * vz;
    }
    if (X) { X[0] = px; X[1] = py; X[2] = pz; }
    const double detJ = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
    *J = detJ;
    const double invJ = 1.0 / detJ;
    met[0] = invJ * (ys * zt - yt * zs);
    met[1] = invJ * (yt * zr - yr * zt);
    met[2] = invJ * (yr * zs - ys * zr);
    met[3] = invJ * (xt * zs - xs * zt);
    met[4] = invJ * (xr * zt - xt * zr);
    met[5] = invJ * (xs * zr - xr * zs);
    met[6] = invJ * (xs * yt - xt * ys);
    met[7] = invJ * (xt * yr - xr * yt);
    met[8] = invJ * (xr * ys - xs * yr);
}

// Per-element geometry of a box cavity, computed from the box parameters with
// the reference's trilinear arithmetic at exactly the nodes the mesh analysis
// samples (node 0 for J^{-T} and J, face point (0,0) for each face's normal and
// lift), so it equals what nwb_box_mesh_create + analysis would produce.
void box_geometry(int N, int nelx, int nely, int nelz, const double lo[3], const double hi[3],
                  int pmask, const std::vector<double>& z, const std::vector<double>& w,
                  std::vector<ElemGeo>& geo, std::vector<int>& conn) {
    const int nelt = nelx * nely * nelz;
    geo.assign(nelt, ElemGeo{});
    conn.assign(6 * static_cast<size_t>(nelt), kConnPEC);
    const double dx = (hi[0] - lo[0]) / nelx, dy = (hi[1] - lo[1]) / nely, dz = (hi[2] - lo[2]) / nelz;
    const int last = N - 1;
    // local (i,j,k) of face point (0,0) of faces 0..5 (src/mesh.cpp:959-976)
    const int fi[6][3] = {{0, 0, 0}, {last, 0, 0}, {0, last, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, last}};
    const double sgn[6] = {-1, 1, 1, -1, -1, 1};
    const int row[6] = {1, 0, 1, 0, 2, 2};  // s, r, s, r, t, t
    auto eidx = [=](int a, int b, int c) { return a + nelx * (b + nely * c); };
    for (int ez = 0; ez < nelz; ++ez)
        for (int ey = 0; ey < nely; ++ey)
            for (int ex = 0; ex < nelx; ++ex) {
                const double x0 = lo[0] + ex * dx, x1 = x0 + dx;
                const double y0 = lo[1] + ey * dy, y1 = y0 + dy;
                const double z0 = lo[2] + ez * dz, z1 = z0 + dz;
                const double c[8][3] = {{x0, y0, z0}, {x1, y0, z0}, {x1, y1, z0}, {x0, y1, z0},
                                        {x0, y0, z1}, {x1, y0, z1}, {x1, y1, z1}, {x0, y1, z1}};
                const int e = eidx(ex, ey, ez);
                ElemGeo& G = geo[e];
                double J0;
                trilinear_point(c, z[0], z[0], z[0], nullptr, &J0, G.met);
                G.jdet = J0;
                for (int f = 0; f < 6; ++f) {
                    double J, met[9];
                    trilinear_point(c, z[fi[f][0]], z[fi[f][1]], z[fi[f][2]], nullptr, &J, met);
                    // row of J^{-T} for the face's reference direction: (r|s|t)_(x,y,z)
                    const double Nx = sgn[f] * J * met[row[f] + 0];
                    const double Ny = sgn[f] * J * met[row[f] + 3];
                    const double Nz = sgn[f] * J * met[row[f] + 6];
                    const double L = std::sqrt(Nx * Nx + Ny * Ny + Nz * Nz);
                    G.nrm[f][0] = (L > 1e-14) ? (Nx / L) : 0.0;
                    G.nrm[f][1] = (L > 1e-14) ? (Ny / L) : 0.0;
                    G.nrm[f][2] = (L > 1e-14) ? (Nz / L) : 0.0;
                    const double dA = L * (w[0] * w[0]);
                    const double w3v = w[fi[f][0]] * w[fi[f][1]] * w[fi[f][2]];
                    G.lift[f] = dA / (J * w3v);
                }
                int nb[6];
                nb[0] = ey > 0 ? eidx(ex, ey - 1, ez) : ((pmask & 2) ? eidx(ex, nely - 1, ez) : -1);
                nb[1] = ex < nelx - 1 ? eidx(ex + 1, ey, ez) : ((pmask & 1) ? eidx(0, ey, ez) : -1);
                nb[2] = ey < nely - 1 ? eidx(ex, ey + 1, ez) : ((pmask & 2) ? eidx(ex, 0, ez) : -1);
                nb[3] = ex > 0 ? eidx(ex - 1, ey, ez) : ((pmask & 1) ? eidx(nelx - 1, ey, ez) : -1);
                nb[4] = ez > 0 ? eidx(ex, ey, ez - 1) : ((pmask & 4) ? eidx(ex, ey, nelz - 1) : -1);
                nb[5] = ez < nelz - 1 ? eidx(ex, ey, ez + 1) : ((pmask & 4) ? eidx(ex, ey, 0) : -1);
                const int opp[6] = {2, 3, 0, 1, 5, 4};
                for (int f = 0; f < 6; ++f)
                    conn[6 * static_cast<size_t>(e) + f] = nb[f] < 0 ? kConnPEC : ((nb[f] << 6) | (opp[f] << 3));
            }
}

// ProbeManager::init (src/probe.cpp:33-96) on a box: first element whose box is
// nearest, reference coordinates clamped to [-1,1], tensor Lagrange weights
// (src/probe.cpp:11-30).
void box_probes(int N, int nelx, int nely, int nelz, const double lo[3], const double hi[3],
                const std::vector<double>& z, int nprobes, const double* xyz, std::vector<int>& elem,
                std::vector<double>& wts) {
    const double h[3] = {(hi[0] - lo[0]) / nelx, (hi[1] - lo[1]) / nely, (hi[2] - lo[2]) / nelz};
    const int nel[3] = {nelx, nely, nelz};
    elem.assign(nprobes, 0);
    wts.assign(static_cast<size_t>(nprobes) * 3 * N, 0.0);
    for (int q = 0; q < nprobes; ++q) {
        // the nearest element per axis, lowest index on ties (argmin over e)
        int best[3];
        double ref[3];
        for (int a = 0; a < 3; ++a) {
            double bd = 1e300;
            int bi = 0;
            double br = 0;
            for (int i = 0; i < nel[a]; ++i) {
                const double x0 = lo[a] + i * h[a], x1 = x0 + h[a];
                const double r = std::abs(x1 - x0) > 1e-14 ? 2.0 * (xyz[3 * q + a] - x0) / (x1 - x0) - 1.0 : 0.0;
                const double d = std::max(0.0, std::max(-1.0 - r, r - 1.0));
                if (d * d < bd) {
                    bd = d * d;
                    bi = i;
                    br = std::max(-1.0, std::min(1.0, r));
                }
            }
            best[a] = bi;
            ref[a] = br;
        }
        elem[q] = best[0] + nelx * (best[1] + nely * best[2]);
        for (int a = 0; a < 3; ++a) {
            double* L = &wts[(static_cast<size_t>(q) * 3 + a) * N];
            int hit = -1;
            for (int i = 0; i < N; ++i)
                if (std::abs(ref[a] - z[i]) < 1e-12) { hit = i; break; }
            for (int i = 0; i < N; ++i) L[i] = hit >= 0 ? (i == hit ? 1.0 : 0.0) : 1.0;
            if (hit >= 0) continue;
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < N; ++j)
                    if (i != j) L[i] *= (ref[a] - z[j]) / (z[i] - z[j]);
        }
    }
}

}  // namespace nwb

namespace {
using nwb::gll;

inline int face_node(int N, int e, int f, int p, int q) {
    int i = 0, j = 0, k = 0;
    switch (f) {
        case 0: i = p; j = 0; k = q; break;
        case 1: i = N - 1; j = p; k = q; break;
        case 2: i = p; j = N - 1; k = q; break;
        case 3: i = 0; j = p; k = q; break;
        case 4: i = p; j = q; k = 0; break;
        default: i = p; j = q; k = N - 1; break;
    }
    return e * N * N * N + i + N * (j + N * k);
}

}  // namespace

extern "C" {

nwb_status nwb_box_mesh_create(int N, int nelx, int nely, int nelz, double xmin, double xmax,
                               double ymin, double ymax, double zmin, double zmax,
                               int periodic_mask, nwb_box_mesh** out) {
    if (!out) { nwb_set_error_("nwb_box_mesh_create: out is null"); return NWB_EINVAL; }
    *out = nullptr;
    if (N < 2 || N > 10 || nelx < 1 || nely < 1 || nelz < 1) {
        nwb_set_error_("nwb_box_mesh_create: need 2 <= N <= 10 and at least one element per axis");
        return NWB_EINVAL;
    }
    const long long nelt_ll = static_cast<long long>(nelx) * nely * nelz;
    const long long npts_ll = nelt_ll * N * N * N;
    if (nelt_ll > (1LL << 25) || npts_ll > 0x7fffffffLL) {
        nwb_set_error_("nwb_box_mesh_create: mesh too large for 32-bit node indices");
        return NWB_EINVAL;
    }
    if (!(xmax > xmin) || !(ymax > ymin) || !(zmax > zmin)) {
        nwb_set_error_("nwb_box_mesh_create: empty box");
        return NWB_EINVAL;
    }
    nwb_box_mesh* m = new (std::nothrow) nwb_box_mesh();
    if (!m) { nwb_set_error_("nwb_box_mesh_create: out of host memory"); return NWB_ENOMEM; }
    try {
        const int nelt = static_cast<int>(nelt_ll);
        const int N3 = N * N * N, NN = N * N;
        const size_t npts = static_cast<size_t>(npts_ll);
        const size_t nfp = static_cast<size_t>(nelt) * 6 * NN;
        m->N = N;
        m->nelt = nelt;
        gll(N, m->z, m->w, m->D);
        m->w3.resize(N3);
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i) m->w3[i + N * (j + N * k)] = m->w[i] * m->w[j] * m->w[k];
        m->x.resize(npts); m->y.resize(npts); m->zc.resize(npts); m->jac.resize(npts);
        for (auto& v : m->met) v.resize(npts);
        const bool px = periodic_mask & 1, py = periodic_mask & 2, pz = periodic_mask & 4;
        const double dx = (xmax - xmin) / nelx, dy = (ymax - ymin) / nely, dz = (zmax - zmin) / nelz;
        const std::vector<double>& zg = m->z;
        auto eidx = [=](int a, int b, int c) { return a + nelx * (b + nely * c); };
        // neighbour (element, face) per face, -1 = PEC (src/mesh.cpp:718-826)
        std::vector<int> nb(6 * static_cast<size_t>(nelt)), nf(6 * static_cast<size_t>(nelt));
        for (int ez = 0; ez < nelz; ++ez) {
            const double z0 = zmin + ez * dz, z1 = z0 + dz;
            for (int ey = 0; ey < nely; ++ey) {
                const double y0 = ymin + ey * dy, y1 = y0 + dy;
                for (int ex = 0; ex < nelx; ++ex) {
                    const double x0 = xmin + ex * dx, x1 = x0 + dx;
                    const int e = eidx(ex, ey, ez);
                    const double c[8][3] = {{x0, y0, z0}, {x1, y0, z0}, {x1, y1, z0}, {x0, y1, z0},
                                            {x0, y0, z1}, {x1, y0, z1}, {x1, y1, z1}, {x0, y1, z1}};
                    // trilinear map and J^{-T} in the reference's operation order
                    for (int k = 0; k < N; ++k) {
                        const double t = zg[k];
                        for (int j = 0; j < N; ++j) {
                            const double s = zg[j];
                            for (int i = 0; i < N; ++i) {
                                const double r = zg[i];
                                const size_t pt = static_cast<size_t>(e) * N3 + i + N * (j + N * k);
                                const double Nf[8] = {
                                    0.125 * (1.0 - r) * (1.0 - s) * (1.0 - t), 0.125 * (1.0 + r) * (1.0 - s) * (1.0 - t),
                                    0.125 * (1.0 + r) * (1.0 + s) * (1.0 - t), 0.125 * (1.0 - r) * (1.0 + s) * (1.0 - t),
                                    0.125 * (1.0 - r) * (1.0 - s) * (1.0 + t), 0.125 * (1.0 + r) * (1.0 - s) * (1.0 + t),
                                    0.125 * (1.0 + r) * (1.0 + s) * (1.0 + t), 0.125 * (1.0 - r) * (1.0 + s) * (1.0 + t)};
                                const double dr[8] = {
                                    -0.125 * (1.0 - s) * (1.0 - t), 0.125 * (1.0 - s) * (1.0 - t),
                                    0.125 * (1.0 + s) * (1.0 - t), -0.125 * (1.0 + s) * (1.0 - t),
                                    -0.125 * (1.0 - s) * (1.0 + t), 0.125 * (1.0 - s) * (1.0 + t),
                                    0.125 * (1.0 + s) * (1.0 + t), -0.125 * (1.0 + s) * (1.0 + t)};
                                const double ds[8] = {
                                    -0.125 * (1.0 - r) * (1.0 - t), -0.125 * (1.0 + r) * (1.0 - t),
                                    0.125 * (1.0 + r) * (1.0 - t), 0.125 * (1.0 - r) * (1.0 - t),
                                    -0.125 * (1.0 - r) * (1.0 + t), -0.125 * (1.0 + r) * (1.0 + t),
                                    0.125 * (1.0 + r) * (1.0 + t), 0.125 * (1.0 - r) * (1.0 + t)};
                                const double dt[8] = {
                                    -0.125 * (1.0 - r) * (1.0 - s), -0.125 * (1.0 + r) * (1.0 - s),
                                    -0.125 * (1.0 + r) * (1.0 + s), -0.125 * (1.0 - r) * (1.0 + s),
                                    0.125 * (1.0 - r) * (1.0 - s), 0.125 * (1.0 + r) * (1.0 - s),
                                    0.125 * (1.0 + r) * (1.0 + s), 0.125 * (1.0 - r) * (1.0 + s)};
                                double X = 0, Y = 0, Z = 0, xr = 0, yr = 0, zr = 0, xs = 0, ys = 0, zs = 0,
                                       xt = 0, yt = 0, zt = 0;
                                for (int a = 0; a < 8; ++a) {
                                    const double vx = c[a][0], vy = c[a][1], vz = c[a][2];
                                    X += Nf[a] * vx; Y += Nf[a] * vy; Z += Nf[a] * vz;
                                    xr += dr[a] * vx; yr += dr[a] * vy; zr += dr[a] * vz;
                                    xs += ds[a] * vx; ys += ds[a] * vy; zs += ds[a] * vz;
                                    xt += dt[a] * vx; yt += dt[a] * vy; zt += dt[a] * vz;
                                }
                                m->x[pt] = X; m->y[pt] = Y; m->zc[pt] = Z;
                                const double detJ = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) +
                                                    xt * (yr * zs - ys * zr);
                                m->jac[pt] = detJ;
                                const double invJ = 1.0 / detJ;
                                m->met[0][pt] = invJ * (ys * zt - yt * zs);
                                m->met[1][pt] = invJ * (yt * zr - yr * zt);
                                m->met[2][pt] = invJ * (yr * zs - ys * zr);
                                m->met[3][pt] = invJ * (xt * zs - xs * zt);
                                m->met[4][pt] = invJ * (xr * zt - xt * zr);
                                m->met[5][pt] = invJ * (xs * zr - xr * zs);
                                m->met[6][pt] = invJ * (xs * yt - xt * ys);
                                m->met[7][pt] = invJ * (xt * yr - xr * yt);
                                m->met[8][pt] = invJ * (xr * ys - xs * yr);
                            }
                        }
                    }
                    int* B = &nb[6 * static_cast<size_t>(e)];
                    int* F = &nf[6 * static_cast<size_t>(e)];
                    auto set = [&](int f, bool inside, bool per, int eIn, int ePer, int fOpp) {
                        if (inside) { B[f] = eIn; F[f] = fOpp; }
                        else if (per) { B[f] = ePer; F[f] = fOpp; }
                        else { B[f] = -1; F[f] = -1; }
                    };
                    set(0, ey > 0, py, ey > 0 ? eidx(ex, ey - 1, ez) : 0, eidx(ex, nely - 1, ez), 2);
                    set(1, ex < nelx - 1, px, ex < nelx - 1 ? eidx(ex + 1, ey, ez) : 0, eidx(0, ey, ez), 3);
                    set(2, ey < nely - 1, py, ey < nely - 1 ? eidx(ex, ey + 1, ez) : 0, eidx(ex, 0, ez), 0);
                    set(3, ex > 0, px, ex > 0 ? eidx(ex - 1, ey, ez) : 0, eidx(nelx - 1, ey, ez), 1);
                    set(4, ez > 0, pz, ez > 0 ? eidx(ex, ey, ez - 1) : 0, eidx(ex, ey, nelz - 1), 5);
                    set(5, ez < nelz - 1, pz, ez < nelz - 1 ? eidx(ex, ey, ez + 1) : 0, eidx(ex, ey, 0), 4);
                }
            }
        }
        // face points in (element, face, q, p) order (src/mesh.cpp:1003-1004)
        m->vmin.resize(nfp); m->vplus.resize(nfp); m->bc.resize(nfp);
        m->nx.resize(nfp); m->ny.resize(nfp); m->nz.resize(nfp); m->dA.resize(nfp);
        const double* rx = m->met[0].data(); const double* sx = m->met[1].data();
        const double* tx = m->met[2].data(); const double* ry = m->met[3].data();
        const double* sy = m->met[4].data(); const double* ty = m->met[5].data();
        const double* rz = m->met[6].data(); const double* sz = m->met[7].data();
        const double* tz = m->met[8].data();
        for (int e = 0; e < nelt; ++e)
            for (int f = 0; f < 6; ++f) {
                const int eB = nb[6 * static_cast<size_t>(e) + f];
                const int fB = nf[6 * static_cast<size_t>(e) + f];
                for (int q = 0; q < N; ++q)
                    for (int p = 0; p < N; ++p) {
                        const size_t fp = (static_cast<size_t>(e) * 6 + f) * NN + q * N + p;
                        const int vM = face_node(N, e, f, p, q);
                        const double J = m->jac[vM];
                        const double w2 = m->w[p] * m->w[q];
                        double Nx = 0, Ny = 0, Nz = 0;
                        switch (f) {
                            case 0: Nx = -J * sx[vM]; Ny = -J * sy[vM]; Nz = -J * sz[vM]; break;
                            case 1: Nx = +J * rx[vM]; Ny = +J * ry[vM]; Nz = +J * rz[vM]; break;
                            case 2: Nx = +J * sx[vM]; Ny = +J * sy[vM]; Nz = +J * sz[vM]; break;
                            case 3: Nx = -J * rx[vM]; Ny = -J * ry[vM]; Nz = -J * rz[vM]; break;
                            case 4: Nx = -J * tx[vM]; Ny = -J * ty[vM]; Nz = -J * tz[vM]; break;
                            default: Nx = +J * tx[vM]; Ny = +J * ty[vM]; Nz = +J * tz[vM]; break;
                        }
                        const double L = std::sqrt(Nx * Nx + Ny * Ny + Nz * Nz);
                        m->nx[fp] = (L > 1e-14) ? (Nx / L) : 0.0;
                        m->ny[fp] = (L > 1e-14) ? (Ny / L) : 0.0;
                        m->nz[fp] = (L > 1e-14) ? (Nz / L) : 0.0;
                        m->dA[fp] = L * w2;
                        m->vmin[fp] = vM;
                        const int vP = eB < 0 ? -1 : face_node(N, eB, fB, p, q);
                        m->vplus[fp] = vP;
                        m->bc[fp] = vP < 0 ? 1 : 0;
                    }
            }
    } catch (const std::bad_alloc&) {
        delete m;
        nwb_set_error_("nwb_box_mesh_create: out of host memory");
        return NWB_ENOMEM;
    }
    *out = m;
    return NWB_OK;
}

nwb_status nwb_box_mesh_desc(const nwb_box_mesh* m, nwb_mesh_desc* d) {
    if (!m || !d) { nwb_set_error_("nwb_box_mesh_desc: null argument"); return NWB_EINVAL; }
    d->N = m->N;
    d->nelt = m->nelt;
    d->D = m->D.data();
    d->w3 = m->w3.data();
    d->jac = m->jac.data();
    for (int c = 0; c < 9; ++c) d->met[c] = m->met[c].data();
    d->vol_idx_minus = m->vmin.data();
    d->vol_idx_plus = m->vplus.data();
    d->bc_type = m->bc.data();
    d->nx = m->nx.data();
    d->ny = m->ny.data();
    d->nz = m->nz.data();
    d->dA = m->dA.data();
    return NWB_OK;
}

nwb_status nwb_box_mesh_coords(const nwb_box_mesh* m, const double** x, const double** y,
                               const double** z) {
    if (!m || !x || !y || !z) { nwb_set_error_("nwb_box_mesh_coords: null argument"); return NWB_EINVAL; }
    *x = m->x.data();
    *y = m->y.data();
    *z = m->zc.data();
    return NWB_OK;
}

nwb_status nwb_box_mesh_gll(const nwb_box_mesh* m, const double** z, const double** w) {
    if (!m || !z || !w) { nwb_set_error_("nwb_box_mesh_gll: null argument"); return NWB_EINVAL; }
    *z = m->z.data();
    *w = m->w.data();
    return NWB_OK;
}

// Mesh::computeMinNodeDistance (src/mesh.cpp:883-930).
nwb_status nwb_box_mesh_dxmin(const nwb_box_mesh* m, double* out) {
    if (!m || !out) { nwb_set_error_("nwb_box_mesh_dxmin: null argument"); return NWB_EINVAL; }
    const int N = m->N;
    const size_t N3 = static_cast<size_t>(N) * N * N;
    double minD2 = 1.0e20;
    for (int e = 0; e < m->nelt; ++e) {
        const size_t off = e * N3;
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i) {
                    const size_t idx = off + i + N * (j + N * k);
                    const size_t nbr[3] = {i + 1 < N ? off + (i + 1) + N * (j + N * k) : idx,
                                           j + 1 < N ? off + i + N * ((j + 1) + N * k) : idx,
                                           k + 1 < N ? off + i + N * (j + N * (k + 1)) : idx};
                    for (size_t q : nbr) {
                        if (q == idx) continue;
                        const double dx = m->x[q] - m->x[idx], dy = m->y[q] - m->y[idx],
                                     dz = m->zc[q] - m->zc[idx];
                        const double d2 = dx * dx + dy * dy + dz * dz;
                        if (d2 < minD2) minD2 = d2;
                    }
                }
    }
    *out = std::sqrt(minD2);
    return NWB_OK;
}

void nwb_box_mesh_destroy(nwb_box_mesh* m) { delete m; }

// ProbeManager::init (src/probe.cpp:33-96) on a box mesh: the probes'
// elements and 1-D Lagrange weights, as the pool locates them.
nwb_status nwb_box_probes(int N, int nelx, int nely, int nelz, double xmin, double xmax, double ymin,
                          double ymax, double zmin, double zmax, int nprobes, const double* xyz,
                          int* elem, double* weights) {
    if (N < 2 || N > 10 || nelx < 1 || nely < 1 || nelz < 1 || nprobes < 0 ||
        (nprobes > 0 && (!xyz || !elem || !weights)) || !(xmax > xmin) || !(ymax > ymin) ||
        !(zmax > zmin)) {
        nwb_set_error_("nwb_box_probes: bad argument");
        return NWB_EINVAL;
    }
    try {
        std::vector<double> z, w, D;
        nwb::gll(N, z, w, D);
        const double lo[3] = {xmin, ymin, zmin}, hi[3] = {xmax, ymax, zmax};
        std::vector<int> el;
        std::vector<double> wt;
        nwb::box_probes(N, nelx, nely, nelz, lo, hi, z, nprobes, xyz, el, wt);
        std::copy(el.begin(), el.end(), elem);
        std::copy(wt.begin(), wt.end(), weights);
    } catch (const std::bad_alloc&) {
        nwb_set_error_("nwb_box_probes: out of host memory");
        return NWB_ENOMEM;
    }
    return NWB_OK;
}

}  // extern "C"
