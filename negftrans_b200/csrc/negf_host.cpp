// negf_host.cpp -- host-side set-up of the engine: the parts of src/grid.f90
// and src/main.f90 that run once per problem (plane-wave basis, k-mesh,
// potential transform) and the plane-wave -> real-space diagonal transform.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "negf_gpu.h"

namespace {
constexpr double PI = 3.141592653589793;  // global.f90:28
using zc = std::complex<double>;

// |G|^2/2 <= ENCUT test of grid.f90:401-402 and 422-423
inline bool in_cutoff(int i, int j, double encut, double lx, double ly) {
    const double gx = (double)(2 * i) * PI / lx, gy = (double)(2 * j) * PI / ly;
    return (gx * gx + gy * gy) / 2 <= encut;
}
inline int nmax(double l, double encut) { return (int)std::ceil(l / PI * std::sqrt(encut / 2)); }

// Twiddle table e^{-2 pi i m / n}, m = 0..n-1.
std::vector<zc> twiddles(int n) {
    std::vector<zc> t(n);
    for (int m = 0; m < n; ++m) {
        const double a = -2.0 * PI * (double)m / n;
        t[m] = zc(std::cos(a), std::sin(a));
    }
    return t;
}
inline int pmod(long long a, int n) {
    long long r = a % n;
    return (int)(r < 0 ? r + n : r);
}
}  // namespace

extern "C" {

int negf_basis_size(double encut, double lx, double ly, int32_t *n) {
    if (!n || !(lx > 0) || !(ly > 0) || !(encut >= 0)) return NEGF_ERR_ARG;
    const int mx = nmax(lx, encut), my = nmax(ly, encut);
    int c = 0;
    for (int j = -my; j <= my; ++j)
        for (int i = -mx; i <= mx; ++i) c += in_cutoff(i, j, encut, lx, ly);
    *n = c;
    return NEGF_OK;
}

int negf_basis(double encut, double lx, double ly, int32_t n, int32_t *nx, int32_t *ny) {
    int32_t want = 0;
    int rc = negf_basis_size(encut, lx, ly, &want);
    if (rc) return rc;
    if (!nx || !ny || n < want) return NEGF_ERR_ARG;
    const int mx = nmax(lx, encut), my = nmax(ly, encut);
    int c = 0;
    // j outer, i inner: the order fixes the matrix layout (grid.f90:420-429)
    for (int j = -my; j <= my; ++j)
        for (int i = -mx; i <= mx; ++i)
            if (in_cutoff(i, j, encut, lx, ly)) { nx[c] = i; ny[c] = j; ++c; }
    return NEGF_OK;
}

// |k+G|^2/2 <= encut around one k-point, enumerated j outer / i inner like
// grid.f90:420-429 (the reference's basis is the k = 0 case).
int negf_basis_k(double encut, double lx, double ly, double kx, double ky, int32_t n, int32_t *count,
                 int32_t *nx, int32_t *ny) {
    if (!count || !(lx > 0) || !(ly > 0) || !(encut >= 0)) return NEGF_ERR_ARG;
    const double gc = std::sqrt(2 * encut);
    const int i0 = (int)std::floor((-gc - kx) * lx / (2 * PI)) - 1, i1 = (int)std::ceil((gc - kx) * lx / (2 * PI)) + 1;
    const int j0 = (int)std::floor((-gc - ky) * ly / (2 * PI)) - 1, j1 = (int)std::ceil((gc - ky) * ly / (2 * PI)) + 1;
    int c = 0;
    for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) {
            const double gx = (double)(2 * i) * PI / lx + kx, gy = (double)(2 * j) * PI / ly + ky;
            if ((gx * gx + gy * gy) / 2 <= encut) {
                if (nx && ny && c < n) { nx[c] = i; ny[c] = j; }
                ++c;
            }
        }
    *count = c;
    if ((nx || ny) && c > n) return NEGF_ERR_ARG;
    return NEGF_OK;
}

int negf_kmesh(int32_t nkx, int32_t nky, double lx, double ly, double *out) {
    if (!out || nkx < 1 || nky < 1) return NEGF_ERR_ARG;
    for (int j = 1; j <= nky; ++j)
        for (int i = 1; i <= nkx; ++i) {
            const int idx = (j - 1) * nkx + (i - 1);
            out[3 * idx + 0] = (i - (1 + nkx) / 2.0) / nkx * (2 * PI / lx);
            out[3 * idx + 1] = (j - (1 + nky) / 2.0) / nky * (2 * PI / ly);
            out[3 * idx + 2] = 1.0 / (nkx * nky);
        }
    return NEGF_OK;
}

// V_reciprocal(i,j) = (1/(Nx Ny)) sum_{x,y} V(x,y) e^{-2 pi i (x i / Nx + y j / Ny)}
// which is what grid.f90:45-68 computes (the (-1)^(y) factor shifts the r2c
// output by Ny/2 and the read-back at j+1+Ny/2 undoes it), evaluated only on
// the |i| <= ngx/2, |j| <= ngy/2 window that main.f90:242-244 keeps.
int negf_vhat(const double *vreal, int32_t Nx, int32_t Ny, int32_t Nz, int32_t ngx, int32_t ngy,
              double *vhat) {
    if (!vreal || !vhat || Nx < 1 || Ny < 1 || Nz < 1 || ngx < 0 || ngy < 0) return NEGF_ERR_ARG;
    if (2 * ngx > Nx || 2 * ngy > Ny) return NEGF_ERR_ARG;  // grid.f90:33-37
    const int W = 2 * ngx + 1, H = 2 * ngy + 1;
    const int hx = ngx / 2, hy = ngy / 2;
    const std::vector<zc> tx = twiddles(Nx), ty = twiddles(Ny);
    zc *out = reinterpret_cast<zc *>(vhat);
    std::memset(vhat, 0, sizeof(zc) * (size_t)W * H * Nz);
    std::vector<zc> X((size_t)(hx + 1) * Ny);
    const double inv = 1.0 / ((double)Nx * Ny);
    for (int k = 0; k < Nz; ++k) {
        const double *v = vreal + (size_t)Nx * Ny * k;
        // transform along x for the non-negative i of the window
        for (int y = 0; y < Ny; ++y)
            for (int i = 0; i <= hx; ++i) {
                zc s = 0.0;
                for (int x = 0; x < Nx; ++x) s += v[x + (size_t)Nx * y] * tx[pmod((long long)x * i, Nx)];
                X[i + (size_t)(hx + 1) * y] = s;
            }
        zc *o = out + (size_t)W * H * k;
        for (int i = 0; i <= hx; ++i)
            for (int j = -hy; j <= hy; ++j) {
                zc s = 0.0;
                for (int y = 0; y < Ny; ++y) s += X[i + (size_t)(hx + 1) * y] * ty[pmod((long long)y * j, Ny)];
                o[(i + ngx) + (size_t)W * (j + ngy)] = s * inv;
            }
        // V(i,j) = conj(V(-i,-j)) for i < 0 (grid.f90:64-68)
        for (int i = -hx; i <= -1; ++i)
            for (int j = -hy; j <= hy; ++j)
                o[(i + ngx) + (size_t)W * (j + ngy)] = std::conj(o[(-i + ngx) + (size_t)W * (-j + ngy)]);
    }
    return NEGF_OK;
}

// diag(u,v) = sum_ab G(a,b) e^{+2 pi i ((nx_a-nx_b) u / Nx + (ny_a-ny_b) v / Ny)}: the
// diagonal that the forward/backward FFT pair of grid.f90:88-133 extracts from
// GreenTensor.  Bin G on the difference n_a - n_b, then one 2-D DFT per slice.
int negf_ptor(const double *g, const int32_t *nx, const int32_t *ny, int32_t N, int32_t Nz_s, int32_t Nx,
              int32_t Ny, double *out) {
    if (!g || !nx || !ny || !out || N < 1 || Nz_s < 1 || Nx < 1 || Ny < 1) return NEGF_ERR_ARG;
    int mx = 0, my = 0;
    for (int a = 0; a < N; ++a) {
        mx = std::max(mx, std::abs(nx[a]));
        my = std::max(my, std::abs(ny[a]));
    }
    const int BX = 4 * mx + 1, BY = 4 * my + 1;
    const std::vector<zc> tx = twiddles(Nx), ty = twiddles(Ny);
    const zc *G = reinterpret_cast<const zc *>(g);
    zc *O = reinterpret_cast<zc *>(out);
    std::vector<zc> bin((size_t)BX * BY), T((size_t)Nx * BY);
    for (int k = 0; k < Nz_s; ++k) {
        std::fill(bin.begin(), bin.end(), zc(0.0));
        const zc *Gk = G + (size_t)N * N * k;
        for (int b = 0; b < N; ++b)
            for (int a = 0; a < N; ++a)
                bin[(nx[a] - nx[b] + 2 * mx) + (size_t)BX * (ny[a] - ny[b] + 2 * my)] += Gk[a + (size_t)N * b];
        // along x: T(u, dy) = sum_dx bin(dx, dy) e^{+2 pi i dx u / Nx}
        for (int dy = 0; dy < BY; ++dy)
            for (int u = 0; u < Nx; ++u) {
                zc s = 0.0;
                for (int dx = 0; dx < BX; ++dx) {
                    const zc b = bin[dx + (size_t)BX * dy];
                    if (b != zc(0.0)) s += b * std::conj(tx[pmod((long long)(dx - 2 * mx) * u, Nx)]);
                }
                T[u + (size_t)Nx * dy] = s;
            }
        zc *Ok = O + (size_t)Nx * Ny * k;
        for (int v = 0; v < Ny; ++v)
            for (int u = 0; u < Nx; ++u) {
                zc s = 0.0;
                for (int dy = 0; dy < BY; ++dy)
                    s += T[u + (size_t)Nx * dy] * std::conj(ty[pmod((long long)(dy - 2 * my) * v, Ny)]);
                Ok[u + (size_t)Nx * v] = s;
            }
    }
    return NEGF_OK;
}

}  // extern "C"
