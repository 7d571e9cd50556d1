// ORACLE — test infrastructure only.
//
// CPU (C++17 + OpenMP) restatement of the chemrust-scf ChFSI path, used as
// the parity checker for the CUDA implementation and as the timed CPU
// baseline.  Nothing in the product links or calls this file; only tests/,
// __graft_entry__.smoke() and bench.py (cpu_baseline / --impl reference) do.
//
// The reference crate's own ChFSI runs only on a GPU through cudarc and its
// physics crate (chemrust-hamiltonian-core) is not vendored, so no reference
// binary can be built here; this restatement follows the reference's algorithm
// step by step (citations per function, paths relative to the reference
// project) and is pinned by the reference's own known-answer tests
// (tests/test_oracle_golden.py).
//
// Conventions: complex interleaved; band-major psi[b*n_pw+g]; grid index
// ix + nx*(iy + ny*iz); unnormalised FFTs (+1 = G->r "inverse", -1 = r->G
// "forward"); H|psi> applies 1/N^3 at the gather.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

using cplx = std::complex<double>;

namespace {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Mixed-radix (2,3,4,5,...) recursive decimation-in-time DFT.
// out[k] = sum_j in[j*stride] * exp(sign * 2 pi i j k / n)
// Role of the cuFFT batched Z2Z transforms (src/device/fft.rs:177-198).
// ---------------------------------------------------------------------------
struct Fft1d {
    int n = 0;
    std::vector<cplx> w;  // w[j] = exp(+2 pi i j / n)
    std::vector<int> radix;
    explicit Fft1d(int n_ = 1) : n(n_) {
        w.resize(n);
        for (int j = 0; j < n; ++j) w[j] = std::polar(1.0, 2.0 * kPi * j / n);
        int m = n;
        for (int r : {4, 2, 3, 5}) {
            while (m % r == 0) { radix.push_back(r); m /= r; }
        }
        for (int r = 7; m > 1; ++r)
            while (m % r == 0) { radix.push_back(r); m /= r; }
    }
    // recursive DIT on sub-problem of length len = n / (product of radices used)
    void rec(const cplx* in, int stride, cplx* out, int len, int level, int sign,
             cplx* tmp) const {
        if (len == 1) { out[0] = in[0]; return; }
        const int r = radix[level];
        const int m = len / r;
        for (int q = 0; q < r; ++q) rec(in + (size_t)q * stride, stride * r, out + q * m, m,
                                         level + 1, sign, tmp);
        const int wstep = n / len;  // omega_len = w[wstep]
        for (int k = 0; k < m; ++k) {
            cplx t[16];
            for (int q = 0; q < r; ++q) {
                int e = (q * k * wstep) % n;
                cplx tw = sign > 0 ? w[e] : std::conj(w[e]);
                t[q] = out[q * m + k] * tw;
            }
            for (int s = 0; s < r; ++s) {
                cplx acc = 0.0;
                for (int q = 0; q < r; ++q) {
                    int e = (int)(((long long)q * s % r) * (n / r) % n);
                    cplx tw = sign > 0 ? w[e] : std::conj(w[e]);
                    acc += t[q] * tw;
                }
                tmp[s] = acc;
            }
            for (int s = 0; s < r; ++s) out[s * m + k] = tmp[s];
        }
    }
    void run(const cplx* in, int stride, cplx* out, int sign) const {
        cplx tmp[16];
        rec(in, stride, out, n, 0, sign, tmp);
    }
};

struct Fft3d {
    int nx, ny, nz;
    Fft1d fx, fy, fz;
    Fft3d(int x, int y, int z) : nx(x), ny(y), nz(z), fx(x), fy(y), fz(z) {}
    // serial 3D transform of one grid (callers parallelise over grids)
    void run(cplx* g, int sign) const {
        int nmax = std::max(nx, std::max(ny, nz));
        std::vector<cplx> a(nmax), b(nmax);
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy) {
                cplx* line = g + (size_t)nx * (iy + (size_t)ny * iz);
                fx.run(line, 1, b.data(), sign);
                std::memcpy(line, b.data(), sizeof(cplx) * nx);
            }
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix) {
                cplx* base = g + ix + (size_t)nx * ny * iz;
                for (int iy = 0; iy < ny; ++iy) a[iy] = base[(size_t)nx * iy];
                fy.run(a.data(), 1, b.data(), sign);
                for (int iy = 0; iy < ny; ++iy) base[(size_t)nx * iy] = b[iy];
            }
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                cplx* base = g + ix + (size_t)nx * iy;
                for (int iz = 0; iz < nz; ++iz) a[iz] = base[(size_t)nx * ny * iz];
                fz.run(a.data(), 1, b.data(), sign);
                for (int iz = 0; iz < nz; ++iz) base[(size_t)nx * ny * iz] = b[iz];
            }
    }
    // parallel 3D transform of one grid
    void run_par(cplx* g, int sign) const {
#pragma omp parallel
        {
            int nmax = std::max(nx, std::max(ny, nz));
            std::vector<cplx> a(nmax), b(nmax);
#pragma omp for collapse(2) schedule(static)
            for (int iz = 0; iz < nz; ++iz)
                for (int iy = 0; iy < ny; ++iy) {
                    cplx* line = g + (size_t)nx * (iy + (size_t)ny * iz);
                    fx.run(line, 1, b.data(), sign);
                    std::memcpy(line, b.data(), sizeof(cplx) * nx);
                }
#pragma omp for collapse(2) schedule(static)
            for (int iz = 0; iz < nz; ++iz)
                for (int ix = 0; ix < nx; ++ix) {
                    cplx* base = g + ix + (size_t)nx * ny * iz;
                    for (int iy = 0; iy < ny; ++iy) a[iy] = base[(size_t)nx * iy];
                    fy.run(a.data(), 1, b.data(), sign);
                    for (int iy = 0; iy < ny; ++iy) base[(size_t)nx * iy] = b[iy];
                }
#pragma omp for collapse(2) schedule(static)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    cplx* base = g + ix + (size_t)nx * iy;
                    for (int iz = 0; iz < nz; ++iz) a[iz] = base[(size_t)nx * ny * iz];
                    fz.run(a.data(), 1, b.data(), sign);
                    for (int iz = 0; iz < nz; ++iz) base[(size_t)nx * ny * iz] = b[iz];
                }
        }
    }
};

// ---------------------------------------------------------------------------
// Dense complex helpers (row-major n x n)
// ---------------------------------------------------------------------------
// Cholesky S = L L^H in place (lower). Returns 0 or the 1-based failing
// column (ZPOTRF info convention; role of faer cholesky_in_place,
// src/eigensolver/subspace_diag.rs:275-292).
int cholesky(std::vector<cplx>& a, int n) {
    for (int j = 0; j < n; ++j) {
        double d = a[(size_t)j * n + j].real();
        for (int k = 0; k < j; ++k) d -= std::norm(a[(size_t)j * n + k]);
        if (!(d > 0.0)) return j + 1;
        double ljj = std::sqrt(d);
        a[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            cplx s = a[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= a[(size_t)i * n + k] * std::conj(a[(size_t)j * n + k]);
            a[(size_t)i * n + j] = s / ljj;
        }
        for (int i = 0; i < j; ++i) a[(size_t)i * n + j] = 0.0;
    }
    return 0;
}

// Inverse of lower-triangular L by forward substitution of L X = I
// (subspace_diag.rs:295-302).
std::vector<cplx> tri_lower_inverse(const std::vector<cplx>& l, int n) {
    std::vector<cplx> x((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        for (int i = c; i < n; ++i) {
            cplx s = (i == c) ? 1.0 : 0.0;
            for (int k = c; k < i; ++k) s -= l[(size_t)i * n + k] * x[(size_t)k * n + c];
            x[(size_t)i * n + c] = s / l[(size_t)i * n + i];
        }
    }
    return x;
}

// Cyclic Jacobi eigen-decomposition of a Hermitian matrix (row-major).
// Eigenvalues ascending; eigenvectors in the columns of v.  Role of faer
// self_adjoint_evd (subspace_diag.rs:335-363).
void jacobi_evd(std::vector<cplx> a, int n, std::vector<double>& w, std::vector<cplx>& v) {
    v.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
    auto A = [&](int i, int j) -> cplx& { return a[(size_t)i * n + j]; };
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double m = std::norm(A(i, j));
                tot += m;
                if (i != j) off += m;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                cplx b = A(p, q);
                double bm = std::abs(b);
                if (bm == 0.0) continue;
                double app = A(p, p).real(), aqq = A(q, q).real();
                cplx ph = b / bm;  // e^{i phi}
                double tau = (aqq - app) / (2.0 * bm);
                double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
                double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
                cplx gqp = -s * std::conj(ph), gqq = c * std::conj(ph);
                // A <- A G (columns p, q)
                for (int k = 0; k < n; ++k) {
                    cplx akp = A(k, p), akq = A(k, q);
                    A(k, p) = akp * c + akq * gqp;
                    A(k, q) = akp * s + akq * gqq;
                }
                // A <- G^H A (rows p, q)
                for (int k = 0; k < n; ++k) {
                    cplx apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk + std::conj(gqp) * aqk;
                    A(q, k) = s * apk + std::conj(gqq) * aqk;
                }
                A(p, q) = 0.0;
                A(q, p) = 0.0;
                A(p, p) = A(p, p).real();
                A(q, q) = A(q, q).real();
                for (int k = 0; k < n; ++k) {
                    cplx vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
                    v[(size_t)k * n + p] = vkp * c + vkq * gqp;
                    v[(size_t)k * n + q] = vkp * s + vkq * gqq;
                }
            }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int x, int y) { return A(x, x).real() < A(y, y).real(); });
    w.resize(n);
    std::vector<cplx> vs((size_t)n * n);
    for (int j = 0; j < n; ++j) {
        w[j] = A(idx[j], idx[j]).real();
        for (int i = 0; i < n; ++i) vs[(size_t)i * n + j] = v[(size_t)i * n + idx[j]];
    }
    v.swap(vs);
}

// Largest eigenvalue of a real symmetric tridiagonal matrix by bisection
// on the Sturm count.
double tridiag_max_eig(const std::vector<double>& d, const std::vector<double>& e) {
    int k = (int)d.size();
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < k; ++i) {
        double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i < k - 1 ? std::fabs(e[i]) : 0.0);
        lo = std::min(lo, d[i] - r);
        hi = std::max(hi, d[i] + r);
    }
    auto count_below = [&](double x) {
        int c = 0;
        double q = d[0] - x;
        if (q < 0) ++c;
        for (int i = 1; i < k; ++i) {
            double qq = q == 0.0 ? 1e-300 : q;
            q = d[i] - x - e[i - 1] * e[i - 1] / qq;
            if (q < 0) ++c;
        }
        return c;
    };
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (count_below(mid) >= k) hi = mid; else lo = mid;
    }
    return hi;
}

// PZ81 LDA (Perdew & Zunger 1981 fit of Ceperley-Alder), unpolarised.
void lda_pz(double rho, double& exc, double& vxc) {
    if (rho < 1e-30) { exc = 0.0; vxc = 0.0; return; }
    const double rs = std::cbrt(3.0 / (4.0 * kPi * rho));
    const double ex = -0.4581652932831429 / rs;
    const double vx = 4.0 / 3.0 * ex;
    double ec, vc;
    if (rs >= 1.0) {
        const double g = -0.1423, b1 = 1.0529, b2 = 0.3334;
        const double sr = std::sqrt(rs);
        const double den = 1.0 + b1 * sr + b2 * rs;
        ec = g / den;
        vc = ec * (1.0 + 7.0 / 6.0 * b1 * sr + 4.0 / 3.0 * b2 * rs) / den;
    } else {
        const double A = 0.0311, B = -0.048, C = 0.0020, D = -0.0116;
        const double lr = std::log(rs);
        ec = A * lr + B + C * rs * lr + D * rs;
        vc = A * lr + (B - A / 3.0) + 2.0 / 3.0 * C * rs * lr + (2.0 * D - C) / 3.0 * rs;
    }
    exc = ex + ec;
    vxc = vx + vc;
}

uint64_t splitmix_next(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

}  // namespace

// ---------------------------------------------------------------------------
// Oracle context
// ---------------------------------------------------------------------------
struct OracleCtx {
    int nx, ny, nz, n_pw, n_bands, n_proj, n_ions;
    double omega, gmax, e_ewald, n_atoms_d;
    Fft3d fft;
    std::vector<int> fft_idx;     // n_pw (scf.rs:387-401)
    std::vector<double> kin;      // n_pw
    std::vector<double> veff;     // N^3
    std::vector<double> vloc_r;   // N^3
    std::vector<cplx> beta;       // n_proj x n_pw
    std::vector<int> poff;        // n_ions + 1
    std::vector<cplx> dmat;       // concatenated ne_i^2 blocks
    std::vector<int> dmat_off;    // n_ions
    std::vector<cplx> psi;        // n_bands x n_pw
    std::vector<cplx> hpsi;       // filtered H psi
    std::vector<double> occ;
    std::vector<double> eig;
    std::vector<double> bounds;   // lambda_max, cut, c, e
    std::vector<double> norms;    // |psi_k| per degree
    int bound_mode = 0, lanczos_steps = 10;
    // ultrasoft overlap S = 1 + beta q beta^H (per-ion q blocks, same layout as D)
    bool uspp = false;
    std::vector<cplx> qmat;
    std::vector<cplx> sinv_m;  // M = q (1 + B q)^-1, B = beta^H beta: S^-1 = 1 - beta M beta^H
    double s_min = 1.0;        // lower bound of the spectrum of S
    // density / mixing state
    std::vector<double> rho_in, rho_out;
    std::vector<std::vector<double>> hist_rho, hist_res;
    OracleCtx(int x, int y, int z) : nx(x), ny(y), nz(z), fft(x, y, z) {}
    size_t ng() const { return (size_t)nx * ny * nz; }
};

namespace {

// out += beta Blk beta^H x for per-ion blocks Blk (D or q), nb vectors.
void add_beta_blocks(const OracleCtx& c, const std::vector<cplx>& blocks, const cplx* x, cplx* out,
                     int nb) {
    if (c.n_proj == 0) return;
    std::vector<cplx> cp((size_t)c.n_proj * nb), cd((size_t)c.n_proj * nb);
#pragma omp parallel for collapse(2) schedule(static)
    for (int p = 0; p < c.n_proj; ++p)
        for (int b = 0; b < nb; ++b) {
            const cplx* bp = &c.beta[(size_t)p * c.n_pw];
            const cplx* ps = x + (size_t)b * c.n_pw;
            cplx s = 0.0;
            for (int g = 0; g < c.n_pw; ++g) s += std::conj(bp[g]) * ps[g];
            cp[(size_t)p * nb + b] = s;
        }
    for (int ion = 0; ion < c.n_ions; ++ion) {
        int p0 = c.poff[ion], ne = c.poff[ion + 1] - p0;
        const cplx* D = &blocks[c.dmat_off[ion]];
        for (int i = 0; i < ne; ++i)
            for (int b = 0; b < nb; ++b) {
                cplx s = 0.0;
                for (int j = 0; j < ne; ++j) s += D[i * ne + j] * cp[(size_t)(p0 + j) * nb + b];
                cd[(size_t)(p0 + i) * nb + b] = s;
            }
    }
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; ++b) {
        cplx* h = out + (size_t)b * c.n_pw;
        for (int g = 0; g < c.n_pw; ++g) {
            cplx s = 0.0;
            for (int p = 0; p < c.n_proj; ++p) s += c.beta[(size_t)p * c.n_pw + g] * cd[(size_t)p * nb + b];
            h[g] += s;
        }
    }
}

// y = S x = x + beta q beta^H x
void apply_s(const OracleCtx& c, const cplx* x, cplx* y, int nb) {
    std::memcpy(y, x, sizeof(cplx) * (size_t)nb * c.n_pw);
    if (c.uspp) add_beta_blocks(c, c.qmat, x, y, nb);
}

// y = S^-1 x = x - beta M beta^H x  (Woodbury with M = q (1 + B q)^-1)
void apply_sinv(const OracleCtx& c, const cplx* x, cplx* y, int nb) {
    std::memcpy(y, x, sizeof(cplx) * (size_t)nb * c.n_pw);
    if (!c.uspp || c.n_proj == 0) return;
    const int np = c.n_proj;
    std::vector<cplx> cp((size_t)np * nb), cm((size_t)np * nb, 0.0);
#pragma omp parallel for collapse(2) schedule(static)
    for (int p = 0; p < np; ++p)
        for (int b = 0; b < nb; ++b) {
            const cplx* bp = &c.beta[(size_t)p * c.n_pw];
            const cplx* ps = x + (size_t)b * c.n_pw;
            cplx s = 0.0;
            for (int g = 0; g < c.n_pw; ++g) s += std::conj(bp[g]) * ps[g];
            cp[(size_t)p * nb + b] = s;
        }
    for (int p = 0; p < np; ++p)
        for (int q = 0; q < np; ++q) {
            const cplx m = c.sinv_m[(size_t)p * np + q];
            if (m == 0.0) continue;
            for (int b = 0; b < nb; ++b) cm[(size_t)p * nb + b] += m * cp[(size_t)q * nb + b];
        }
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; ++b) {
        cplx* h = y + (size_t)b * c.n_pw;
        for (int g = 0; g < c.n_pw; ++g) {
            cplx s = 0.0;
            for (int p = 0; p < np; ++p) s += c.beta[(size_t)p * c.n_pw + g] * cm[(size_t)p * nb + b];
            h[g] -= s;
        }
    }
}

// Inverse of a dense complex matrix by Gauss-Jordan with partial pivoting.
bool invert(std::vector<cplx>& a, int n) {
    std::vector<cplx> inv((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (std::abs(a[(size_t)r * n + col]) > std::abs(a[(size_t)piv * n + col])) piv = r;
        if (std::abs(a[(size_t)piv * n + col]) == 0.0) return false;
        if (piv != col)
            for (int k = 0; k < n; ++k) {
                std::swap(a[(size_t)col * n + k], a[(size_t)piv * n + k]);
                std::swap(inv[(size_t)col * n + k], inv[(size_t)piv * n + k]);
            }
        const cplx d = a[(size_t)col * n + col];
        for (int k = 0; k < n; ++k) { a[(size_t)col * n + k] /= d; inv[(size_t)col * n + k] /= d; }
#pragma omp parallel for schedule(static) if (n > 256)
        for (int r = 0; r < n; ++r) {
            if (r == col) continue;
            const cplx f = a[(size_t)r * n + col];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                a[(size_t)r * n + k] -= f * a[(size_t)col * n + k];
                inv[(size_t)r * n + k] -= f * inv[(size_t)col * n + k];
            }
        }
    }
    a.swap(inv);
    return true;
}

// H|psi> = T psi + (1/N^3) FFT[-1]( V .* FFT[+1](scatter psi) ) + beta D beta^H psi
// Order of operations follows apply_v_loc_hamiltonian (chebyshev.rs:279-365):
// init_kinetic, zero, scatter, inverse FFT, veff_multiply, forward FFT,
// gather_add (x 1/N^3); then apply_v_nl_hamiltonian (chebyshev.rs:416-500):
// C = beta^H psi, C = D C, Hpsi += beta C.
void apply_h(const OracleCtx& c, const cplx* psi, cplx* hpsi, int nb) {
    const size_t ng = c.ng();
    const double inv_n = 1.0 / (double)ng;
#pragma omp parallel
    {
        std::vector<cplx> grid(ng);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nb; ++b) {
            const cplx* p = psi + (size_t)b * c.n_pw;
            cplx* h = hpsi + (size_t)b * c.n_pw;
            for (int g = 0; g < c.n_pw; ++g) h[g] = p[g] * c.kin[g];
            std::fill(grid.begin(), grid.end(), cplx(0.0));
            for (int g = 0; g < c.n_pw; ++g) grid[c.fft_idx[g]] = p[g];
            c.fft.run(grid.data(), +1);
            for (size_t r = 0; r < ng; ++r) grid[r] *= c.veff[r];
            c.fft.run(grid.data(), -1);
            for (int g = 0; g < c.n_pw; ++g) h[g] += grid[c.fft_idx[g]] * inv_n;
        }
    }
    add_beta_blocks(c, c.dmat, psi, hpsi, nb);
}

double frob_norm(const std::vector<cplx>& x) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s)
    for (size_t i = 0; i < x.size(); ++i) s += std::norm(x[i]);
    return std::sqrt(s);
}

// Deterministic Lanczos start vector shared with the device implementation:
// SplitMix64(seed 0x5EED) uniform pairs mapped to [-1/2, 1/2).
void lanczos_start(std::vector<cplx>& v, int n) {
    uint64_t s = 0x5EEDULL;
    v.resize(n);
    for (int g = 0; g < n; ++g) {
        double re = (double)(splitmix_next(s) >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        double im = (double)(splitmix_next(s) >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        v[g] = cplx(re, im);
    }
}

// k-step Lanczos upper bound lambda_max(T_k) + |f_k| (Zhou 2010; the
// deferred bound of notes/pr-reviews/phase-2/deferred.md:131-161).
double lanczos_upper(const OracleCtx& c, int k) {
    const int n = c.n_pw;
    std::vector<cplx> v, v0(n, 0.0), f(n);
    lanczos_start(v, n);
    double nv = 0.0;
    for (auto& x : v) nv += std::norm(x);
    nv = std::sqrt(nv);
    for (auto& x : v) x /= nv;
    std::vector<double> d, e;
    double beta = 0.0;
    for (int j = 0; j < k; ++j) {
        apply_h(c, v.data(), f.data(), 1);
        if (j > 0)
            for (int g = 0; g < n; ++g) f[g] -= beta * v0[g];
        double alpha = 0.0;
        for (int g = 0; g < n; ++g) alpha += (std::conj(v[g]) * f[g]).real();
        for (int g = 0; g < n; ++g) f[g] -= alpha * v[g];
        d.push_back(alpha);
        double fn = 0.0;
        for (int g = 0; g < n; ++g) fn += std::norm(f[g]);
        fn = std::sqrt(fn);
        if (j == k - 1) {
            return tridiag_max_eig(d, e) + fn;
        }
        e.push_back(fn);
        beta = fn;
        v0 = v;
        for (int g = 0; g < n; ++g) v[g] = f[g] / fn;
    }
    return 0.0;
}

// Fermi-Dirac occupations f_i = 2 / (1 + exp((e_i - mu)/kT)) with mu from
// bisection on sum f = n_elec (construct_density's planned occupation step,
// PROJECT_ROOT_PLAN.md:582-589, SmearingParams src/types.rs:204-211).
// kT <= 0: aufbau (f = 2 for the lowest n_elec/2 bands).  Returns -kT S, the
// entropy term of the free energy.
double fermi_occupations(const double* e, int n, double n_elec, double kT, double* f) {
    if (kT <= 0.0) {
        double left = n_elec;
        for (int i = 0; i < n; ++i) {
            f[i] = std::min(2.0, std::max(0.0, left));
            left -= f[i];
        }
        return 0.0;
    }
    double lo = e[0], hi = e[0];
    for (int i = 0; i < n; ++i) { lo = std::min(lo, e[i]); hi = std::max(hi, e[i]); }
    lo -= 40.0 * kT + 1.0;
    hi += 40.0 * kT + 1.0;
    auto count = [&](double mu) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
            double x = std::min(700.0, std::max(-700.0, (e[i] - mu) / kT));
            s += 2.0 / (1.0 + std::exp(x));
        }
        return s;
    };
    for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (count(mid) < n_elec) lo = mid; else hi = mid;
    }
    const double mu = 0.5 * (lo + hi);
    double ts = 0.0;
    for (int i = 0; i < n; ++i) {
        double x = std::min(700.0, std::max(-700.0, (e[i] - mu) / kT));
        f[i] = 2.0 / (1.0 + std::exp(x));
        double ft = 0.5 * f[i];
        if (ft > 1e-300 && ft < 1.0 - 1e-16) ts += -2.0 * (ft * std::log(ft) + (1.0 - ft) * std::log(1.0 - ft));
    }
    return -kT * ts;
}

}  // namespace

// ---------------------------------------------------------------------------
// Band-by-band preconditioned CG refinement (src/eigensolver/band_cg.rs:157-437)
// with the closed-form 2x2 line search (line_search.rs:57-212), residual /
// S-orthogonalisation helpers (cg_helpers.rs:49-216) and the TPA + ultrasoft
// Woodbury preconditioner (uspp_preconditioner.rs:56-300).
// ---------------------------------------------------------------------------
struct LineSearch { double step, eig, norm; int status; };

LineSearch line_search_2d(double a, double hpsi_dir, double c, double d) {
    const double b = -2.0 * hpsi_dir;
    double step = 0.0, eig = a;
    int status = 0;
    if (std::fabs(d) > 2.2250738585072014e-308) {
        const double ad = a * d, bd = b * d;
        if (std::fabs(bd) < 1e-30) return {0.0, a, 1.0, -2};
        const double tmp = ad * ad - 2.0 * ad * c + c * c + b * bd;
        if (tmp < 0.0) return {0.0, a, 1.0, -1};
        const double det = std::sqrt(tmp);
        const double r1 = (-ad + c + det) / bd, r2 = (-ad + c - det) / bd;
        auto e_at = [&](double r, bool& ok) {
            const double den = 1.0 + d * r * r;
            ok = den > 0.0;
            return ok ? (a + b * r + c * r * r) / den : 0.0;
        };
        bool ok1, ok2;
        const double e1 = e_at(r1, ok1), e2 = e_at(r2, ok2);
        double rr, ee;
        if (ok1 && ok2) { if (e1 < e2) { rr = r1; ee = e1; } else { rr = r2; ee = e2; } }
        else if (ok1 && e1 < a) { rr = r1; ee = e1; }
        else if (ok2 && e2 < a) { rr = r2; ee = e2; }
        else return {0.0, a, 1.0, -1};
        step = -rr;
        eig = ee;
    } else {
        if (c > 0.0) {
            step = -b / (2.0 * c);
            eig = (a + b * step + c * step * step) / (1.0 + d * step * step);
        } else {
            return {0.0, a, 1.0, -1};
        }
    }
    if (step > 15.0) {
        step = 15.0;
        eig = (a + b * step + c * step * step) / (1.0 + d * step * step);
        status = 1;
    } else if (step < 0.0) {
        status = -1;
    }
    const double t = 1.0 + d * step * step;
    if (t > 0.0) return {step, eig, std::sqrt(t), status};
    return {step, eig, 0.0, 2};
}

// TPA diagonal 1 / (1 + 16 x^4 / (27 + 18 x + 12 x^2 + 8 x^3)), x = E_k / <E_k>
void tpa_diag(const double* kin, int n, double* out) {
    double s = 0.0;
    for (int g = 0; g < n; ++g) s += kin[g];
    const double mean = n > 0 ? s / n : 0.0;
    const double inv = mean > 0.0 ? 1.0 / mean : 1.0;
    for (int g = 0; g < n; ++g) {
        const double x = kin[g] * inv;
        const double den = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
        out[g] = 1.0 / (1.0 + 16.0 * x * x * x * x / den);
    }
}

extern "C" {

}  // extern "C"

namespace {

cplx dotc(const cplx* a, const cplx* b, int n) {
    cplx s = 0.0;
    for (int i = 0; i < n; ++i) s += std::conj(a[i]) * b[i];
    return s;
}

// Preconditioner P^-1 r = T r + T beta R beta^H T r with R = (-q^-1 - beta^H T beta)^-1
// (uspp_preconditioner.rs:80-131, 180-300); without q it is the TPA diagonal.
struct Precond {
    std::vector<double> t;
    std::vector<cplx> r;  // n_proj x n_proj, empty: TPA only
};

Precond build_precond(const OracleCtx& c) {
    Precond P;
    P.t.resize(c.n_pw);
    tpa_diag(c.kin.data(), c.n_pw, P.t.data());
    if (!c.uspp || c.n_proj == 0) return P;
    const int np = c.n_proj;
    std::vector<cplx> Q((size_t)np * np, 0.0), Cm((size_t)np * np);
    for (int ion = 0; ion < c.n_ions; ++ion) {
        const int p0 = c.poff[ion], ne = c.poff[ion + 1] - p0;
        for (int i = 0; i < ne; ++i)
            for (int j = 0; j < ne; ++j) Q[(size_t)(p0 + i) * np + p0 + j] = c.qmat[c.dmat_off[ion] + i * ne + j];
    }
    if (!invert(Q, np)) return P;
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < np; ++p)
        for (int q = 0; q < np; ++q) {
            cplx s = 0.0;
            for (int g = 0; g < c.n_pw; ++g)
                s += std::conj(c.beta[(size_t)p * c.n_pw + g]) * P.t[g] * c.beta[(size_t)q * c.n_pw + g];
            Cm[(size_t)p * np + q] = s;
        }
    std::vector<cplx> M((size_t)np * np);
    for (size_t i = 0; i < M.size(); ++i) M[i] = -Q[i] - Cm[i];
    if (!invert(M, np)) return P;
    P.r = M;
    return P;
}

void apply_precond(const OracleCtx& c, const Precond& P, const cplx* r, cplx* out) {
    const int n = c.n_pw;
    std::vector<cplx> tr(n);
    for (int g = 0; g < n; ++g) tr[g] = r[g] * P.t[g];
    if (P.r.empty()) { std::copy(tr.begin(), tr.end(), out); return; }
    const int np = c.n_proj;
    std::vector<cplx> w(np), wr(np, 0.0);
    for (int p = 0; p < np; ++p) w[p] = dotc(&c.beta[(size_t)p * n], tr.data(), n);
    for (int i = 0; i < np; ++i)
        for (int j = 0; j < np; ++j) wr[i] += P.r[(size_t)i * np + j] * w[j];
    for (int g = 0; g < n; ++g) {
        cplx s = 0.0;
        for (int p = 0; p < np; ++p) s += c.beta[(size_t)p * n + g] * wr[p];
        out[g] = tr[g] + s * P.t[g];
    }
}

struct CgOut { double eig; int steps; bool converged; double rnorm; };

// band_cg_minimize (band_cg.rs:157-437) for one band; psi is replaced by the
// S-normalised refined band.  lower: (psi_j, S psi_j) of the refined lower bands.
CgOut band_cg_one(const OracleCtx& c, const Precond& P, std::vector<cplx>& psi,
                  const std::vector<std::pair<std::vector<cplx>, std::vector<cplx>>>& lower,
                  int max_steps, double tol) {
    const int n = c.n_pw;
    std::vector<cplx> hpsi(n), spsi(n);
    auto apply_hs = [&](const std::vector<cplx>& x, std::vector<cplx>& hx, std::vector<cplx>& sx) {
        apply_h(c, x.data(), hx.data(), 1);
        apply_s(c, x.data(), sx.data(), 1);
    };
    apply_hs(psi, hpsi, spsi);
    const double s0 = dotc(psi.data(), spsi.data(), n).real();
    const double inv0 = 1.0 / std::sqrt(s0);
    for (int g = 0; g < n; ++g) { psi[g] *= inv0; hpsi[g] *= inv0; spsi[g] *= inv0; }
    double eig = dotc(psi.data(), hpsi.data(), n).real();
    auto residual = [&](std::vector<cplx>& r) {
        const double he = dotc(psi.data(), hpsi.data(), n).real();
        const double se = dotc(psi.data(), spsi.data(), n).real();
        const double e = he / se;
        for (int g = 0; g < n; ++g) r[g] = hpsi[g] - e * spsi[g];
    };
    auto norm = [&](const std::vector<cplx>& v) {
        double s = 0.0;
        for (auto& x : v) s += std::norm(x);
        return std::sqrt(s);
    };
    std::vector<cplx> r(n), g(n), sg(n), d(n), d_old, hd(n), sd(n);
    residual(r);
    double beta_old = 0.0;
    for (int step = 1; step <= max_steps; ++step) {
        apply_precond(c, P, r.data(), g.data());
        if (norm(g) < 2.220446049250313e-16 * 1000.0) return {eig, step - 1, true, norm(r)};
        const double prev = eig;
        apply_s(c, g.data(), sg.data(), 1);
        // S-orthogonalise g against the refined lower bands (modified
        // Gram-Schmidt, s_orthogonalize_against, cg_helpers.rs:161-216), then
        // S-normalise.  The reference keeps only Re<psi_j|S|g>
        // (cg_helpers.rs:189), which is the whole overlap for the real-valued
        // Gamma-point bands it targets; with general complex bands that drops
        // Im<psi_j|S|g> and lets the refined bands collapse onto lower ones,
        // so the full complex overlap is removed here.
        for (auto& lb : lower) {
            const cplx ov = dotc(lb.first.data(), sg.data(), n);
            for (int i = 0; i < n; ++i) { g[i] -= ov * lb.first[i]; sg[i] -= ov * lb.second[i]; }
        }
        const double gn = std::sqrt(std::max(dotc(g.data(), sg.data(), n).real(), 1e-300));
        for (int i = 0; i < n; ++i) { g[i] /= gn; sg[i] /= gn; }
        if (step <= 2) {
            d = g;
            beta_old = dotc(g.data(), r.data(), n).real();
        } else {
            const double beta = dotc(g.data(), r.data(), n).real();
            const double gamma = std::fabs(beta_old) > 1e-300 ? beta / beta_old : 0.0;
            for (int i = 0; i < n; ++i) d[i] = gamma * d_old[i] - g[i];
            beta_old = beta;
        }
        apply_hs(d, hd, sd);
        const cplx ov = dotc(psi.data(), sd.data(), n);
        if (std::abs(ov) > 1e-30)
            for (int i = 0; i < n; ++i) { d[i] -= ov * psi[i]; hd[i] -= ov * hpsi[i]; sd[i] -= ov * spsi[i]; }
        d_old = d;
        const double rn = norm(r);
        if (rn < tol * 0.01 && rn < 1e-12 * std::max(std::fabs(eig), 1.0)) return {eig, step - 1, true, rn};
        const LineSearch ls = line_search_2d(eig, dotc(hpsi.data(), d.data(), n).real(),
                                             dotc(hd.data(), d.data(), n).real(),
                                             dotc(sd.data(), d.data(), n).real());
        const double inv = ls.norm > 0.0 ? 1.0 / ls.norm : 1.0;
        for (int i = 0; i < n; ++i) {
            psi[i] = (psi[i] + ls.step * d[i]) * inv;
            hpsi[i] = (hpsi[i] + ls.step * hd[i]) * inv;
            spsi[i] = (spsi[i] + ls.step * sd[i]) * inv;
        }
        const double e_new = dotc(psi.data(), hpsi.data(), n).real();
        residual(r);
        if (std::fabs(e_new - prev) < tol) return {e_new, step, true, norm(r)};
        eig = e_new;
    }
    return {eig, max_steps, false, norm(r)};
}

}  // namespace

extern "C" {

// Refine every band in turn with band_cg_minimize against the already
// refined lower bands (the gate tests' driver, tests/phase0_gate2_convergence.rs:387-418).
// eig_out[b], steps_out[b] per band; returns the number of converged bands.
int oracle_band_cg(OracleCtx* c, int max_steps, double tol, double* eig_out, int* steps_out) {
    const Precond P = build_precond(*c);
    const int n = c->n_pw;
    std::vector<std::pair<std::vector<cplx>, std::vector<cplx>>> lower;
    int nconv = 0;
    for (int b = 0; b < c->n_bands; ++b) {
        std::vector<cplx> psi(c->psi.begin() + (size_t)b * n, c->psi.begin() + (size_t)(b + 1) * n);
        const CgOut o = band_cg_one(*c, P, psi, lower, max_steps, tol);
        std::copy(psi.begin(), psi.end(), c->psi.begin() + (size_t)b * n);
        std::vector<cplx> sp(n);
        apply_s(*c, psi.data(), sp.data(), 1);
        lower.emplace_back(psi, sp);
        if (eig_out) eig_out[b] = o.eig;
        if (steps_out) steps_out[b] = o.steps;
        nconv += o.converged;
    }
    return nconv;
}

void oracle_line_search(double a, double hpsi_dir, double c, double d, double* out4) {
    const LineSearch r = line_search_2d(a, hpsi_dir, c, d);
    out4[0] = r.step; out4[1] = r.eig; out4[2] = r.norm; out4[3] = r.status;
}

void oracle_tpa_diag(const double* kin, int n, double* out) { tpa_diag(kin, n, out); }

double oracle_fermi(const double* e, int n, double n_elec, double kT, double* f) {
    return fermi_occupations(e, n, n_elec, kT, f);
}

OracleCtx* oracle_create(int nx, int ny, int nz, int n_pw, int n_bands, int n_proj, int n_ions,
                         double omega, double gmax, double e_ewald, int n_atoms,
                         const int32_t* miller, const double* kinetic, const double* beta,
                         const int32_t* poff, const double* dmat, const double* psi,
                         const double* occ, const double* vloc_g) {
    OracleCtx* c = new OracleCtx(nx, ny, nz);
    c->n_pw = n_pw; c->n_bands = n_bands; c->n_proj = n_proj; c->n_ions = n_ions;
    c->omega = omega; c->gmax = gmax; c->e_ewald = e_ewald; c->n_atoms_d = n_atoms;
    c->fft_idx.resize(n_pw);
    for (int g = 0; g < n_pw; ++g) {
        int h = miller[3 * g], k = miller[3 * g + 1], l = miller[3 * g + 2];
        int ix = h >= 0 ? h : h + nx, iy = k >= 0 ? k : k + ny, iz = l >= 0 ? l : l + nz;
        c->fft_idx[g] = ix + nx * (iy + ny * iz);
    }
    c->kin.assign(kinetic, kinetic + n_pw);
    c->beta.resize((size_t)n_proj * n_pw);
    if (n_proj) std::memcpy(c->beta.data(), beta, sizeof(cplx) * c->beta.size());
    c->poff.assign(poff, poff + (n_ions > 0 ? n_ions + 1 : 0));
    size_t dtot = 0;
    for (int i = 0; i < n_ions; ++i) {
        c->dmat_off.push_back((int)dtot);
        int ne = c->poff[i + 1] - c->poff[i];
        dtot += (size_t)ne * ne;
    }
    c->dmat.resize(dtot);
    if (dtot) std::memcpy(c->dmat.data(), dmat, sizeof(cplx) * dtot);
    c->psi.resize((size_t)n_bands * n_pw);
    std::memcpy(c->psi.data(), psi, sizeof(cplx) * c->psi.size());
    c->occ.assign(occ, occ + n_bands);
    c->veff.assign(c->ng(), 0.0);
    c->vloc_r.assign(c->ng(), 0.0);
    if (vloc_g) {
        std::vector<cplx> g(c->ng());
        std::memcpy(g.data(), vloc_g, sizeof(cplx) * g.size());
        c->fft.run_par(g.data(), +1);
        for (size_t r = 0; r < c->ng(); ++r) c->vloc_r[r] = g[r].real();
    }
    return c;
}

void oracle_destroy(OracleCtx* c) { delete c; }

int oracle_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void oracle_set_veff(OracleCtx* c, const double* v) { c->veff.assign(v, v + c->ng()); }
// screened D (same block layout as at creation) and occupations, for SCF
// loops driven from Python (ultrasoft augmentation)
void oracle_set_dmat(OracleCtx* c, const double* dmat) {
    std::memcpy(c->dmat.data(), dmat, sizeof(cplx) * c->dmat.size());
}
void oracle_set_occ(OracleCtx* c, const double* occ) { c->occ.assign(occ, occ + c->n_bands); }

// Ultrasoft overlap: per-ion q blocks (layout of D).  Builds the Woodbury
// factor M = q (1 + B q)^-1 with B = beta^H beta and the lower bound
// s_min = 1 - max_i sum_j |(q B)_ij| of the spectrum of S.  Returns 0 or -6.
// bmat: B = beta^H beta (n_proj x n_proj) when the caller has it (a BLAS
// product on the host), else null and formed here.
int oracle_set_qmat_b(OracleCtx* c, const double* qmat, const double* bmat) {
    const int np = c->n_proj;
    c->qmat.assign(c->dmat.size(), 0.0);
    if (np == 0) return -6;
    std::memcpy(c->qmat.data(), qmat, sizeof(cplx) * c->qmat.size());
    std::vector<cplx> Q((size_t)np * np, 0.0), B((size_t)np * np), QB((size_t)np * np, 0.0);
    for (int ion = 0; ion < c->n_ions; ++ion) {
        const int p0 = c->poff[ion], ne = c->poff[ion + 1] - p0;
        for (int i = 0; i < ne; ++i)
            for (int j = 0; j < ne; ++j) Q[(size_t)(p0 + i) * np + p0 + j] = c->qmat[c->dmat_off[ion] + i * ne + j];
    }
    if (bmat) {
        std::memcpy(B.data(), bmat, sizeof(cplx) * B.size());
    } else {
#pragma omp parallel for schedule(dynamic, 1)
        for (int p = 0; p < np; ++p)
            for (int q = 0; q < np; ++q) {
                cplx s = 0.0;
                for (int g = 0; g < c->n_pw; ++g) s += std::conj(c->beta[(size_t)p * c->n_pw + g]) * c->beta[(size_t)q * c->n_pw + g];
                B[(size_t)p * np + q] = s;
            }
    }
    for (int i = 0; i < np; ++i)
        for (int k = 0; k < np; ++k) {
            const cplx qik = Q[(size_t)i * np + k];
            if (qik == 0.0) continue;
            for (int j = 0; j < np; ++j) QB[(size_t)i * np + j] += qik * B[(size_t)k * np + j];
        }
    double rs = 0.0;
    for (int i = 0; i < np; ++i) {
        double r = 0.0;
        for (int j = 0; j < np; ++j) r += std::abs(QB[(size_t)i * np + j]);
        rs = std::max(rs, r);
    }
    c->s_min = std::max(0.1, 1.0 - rs);
    // (1 + B q)^-1
    std::vector<cplx> A((size_t)np * np, 0.0);
    for (int i = 0; i < np; ++i)
        for (int k = 0; k < np; ++k) {
            const cplx bik = B[(size_t)i * np + k];
            if (bik == 0.0) continue;
            for (int j = 0; j < np; ++j) A[(size_t)i * np + j] += bik * Q[(size_t)k * np + j];
        }
    for (int i = 0; i < np; ++i) A[(size_t)i * np + i] += 1.0;
    if (!invert(A, np)) return -6;
    c->sinv_m.assign((size_t)np * np, 0.0);
    for (int i = 0; i < np; ++i)
        for (int k = 0; k < np; ++k) {
            const cplx qik = Q[(size_t)i * np + k];
            if (qik == 0.0) continue;
            for (int j = 0; j < np; ++j) c->sinv_m[(size_t)i * np + j] += qik * A[(size_t)k * np + j];
        }
    c->uspp = true;
    return 0;
}
int oracle_set_qmat(OracleCtx* c, const double* qmat) { return oracle_set_qmat_b(c, qmat, nullptr); }

void oracle_apply_s(OracleCtx* c, const double* x, double* y, int nb) {
    apply_s(*c, reinterpret_cast<const cplx*>(x), reinterpret_cast<cplx*>(y), nb);
}
void oracle_apply_sinv(OracleCtx* c, const double* x, double* y, int nb) {
    apply_sinv(*c, reinterpret_cast<const cplx*>(x), reinterpret_cast<cplx*>(y), nb);
}
double oracle_s_min(OracleCtx* c) { return c->s_min; }
void oracle_get_veff(OracleCtx* c, double* v) { std::memcpy(v, c->veff.data(), sizeof(double) * c->ng()); }
void oracle_get_vloc_r(OracleCtx* c, double* v) { std::memcpy(v, c->vloc_r.data(), sizeof(double) * c->ng()); }
void oracle_set_psi(OracleCtx* c, const double* p) { std::memcpy(c->psi.data(), p, sizeof(cplx) * c->psi.size()); }
void oracle_get_psi(OracleCtx* c, double* p) { std::memcpy(p, c->psi.data(), sizeof(cplx) * c->psi.size()); }
void oracle_get_hpsi(OracleCtx* c, double* p) { std::memcpy(p, c->hpsi.data(), sizeof(cplx) * c->hpsi.size()); }
void oracle_set_bound_mode(OracleCtx* c, int mode, int k) { c->bound_mode = mode; c->lanczos_steps = k; }
void oracle_get_bounds(OracleCtx* c, double* out4) { for (int i = 0; i < 4 && i < (int)c->bounds.size(); ++i) out4[i] = c->bounds[i]; }
int oracle_get_norms(OracleCtx* c, double* out, int n) {
    int m = std::min(n, (int)c->norms.size());
    for (int i = 0; i < m; ++i) out[i] = c->norms[i];
    return (int)c->norms.size();
}

// 3D FFT of one grid in place (exposed for the FFT known-answer tests).
void oracle_fft3d(int nx, int ny, int nz, double* grid, int sign) {
    Fft3d f(nx, ny, nz);
    f.run_par(reinterpret_cast<cplx*>(grid), sign);
}

void oracle_apply_h(OracleCtx* c, const double* psi, double* hpsi, int nb) {
    apply_h(*c, reinterpret_cast<const cplx*>(psi), reinterpret_cast<cplx*>(hpsi), nb);
}

// Spectral bounds (chebyshev.rs:225-254), with the Lanczos upper bound as
// the alternative lambda_max.
void oracle_spectral_bounds(OracleCtx* c, const double* eig, int n_eig, double* out4) {
    double minv = 1e300, maxv = -1e300;
    for (double v : c->veff) { minv = std::min(minv, v); maxv = std::max(maxv, v); }
    double lm;
    if (c->bound_mode == 1) lm = lanczos_upper(*c, c->lanczos_steps);
    else lm = 0.5 * c->gmax * c->gmax + (maxv - minv);
    // generalised problem: the spectrum of S^-1 H lies below lambda_max(H) / lambda_min(S)
    if (c->uspp) lm /= c->s_min;
    double cut;
    if (!eig || n_eig == 0) cut = lm / 3.0;
    else {
        double e0 = eig[0], el = eig[n_eig - 1];
        cut = std::min(el + 0.2 * (el - e0), lm * 0.95);
    }
    out4[0] = lm; out4[1] = cut; out4[2] = (lm + cut) / 2.0; out4[3] = (lm - cut) / 2.0;
}

// Chebyshev filter (chebyshev.rs:626-816): unscaled three-term recurrence
// psi_1 = sigma psi_0, psi_k = 2 sigma psi_{k-1} - psi_{k-2},
// sigma x = (H x)(1/e) + (-c/e) x  (zscal then zaxpy, chebyshev.rs:507-539),
// 10x norm-growth guard (chebyshev.rs:552-563), final H psi for RR.
// Returns 0, or -3 (ChebyshevDiverged) with the failing degree in *fail_k.
int oracle_chebyshev_filter(OracleCtx* c, int ndeg, const double* eig, int n_eig, int* fail_k) {
    double b4[4];
    oracle_spectral_bounds(c, eig, n_eig, b4);
    c->bounds.assign(b4, b4 + 4);
    const double inv_e = 1.0 / b4[3];
    const double ncoe = -b4[2] / b4[3];
    const size_t n = c->psi.size();
    std::vector<cplx> a = c->psi, bb(n), h(n);
    c->norms.clear();
    c->norms.push_back(frob_norm(a));
    if (fail_k) *fail_k = 0;
    int status = 0;
    std::vector<cplx> hs(c->uspp ? n : 0);
    auto op = [&](const cplx* x, cplx* y) {  // y = H x, or S^-1 H x for the generalised problem
        if (!c->uspp) { apply_h(*c, x, y, c->n_bands); return; }
        apply_h(*c, x, hs.data(), c->n_bands);
        apply_sinv(*c, hs.data(), y, c->n_bands);
    };
    if (ndeg >= 1) {
        op(a.data(), h.data());
#pragma omp parallel for
        for (size_t i = 0; i < n; ++i) bb[i] = h[i] * inv_e + ncoe * a[i];
        c->norms.push_back(frob_norm(bb));
    }
    for (int k = 2; k <= ndeg; ++k) {
        op(bb.data(), h.data());
#pragma omp parallel for
        for (size_t i = 0; i < n; ++i) {
            cplx s = h[i] * inv_e + ncoe * bb[i];
            a[i] = 2.0 * s - a[i];  // psi_k overwrites psi_{k-2}
        }
        std::swap(a, bb);  // a = psi_{k-1}, bb = psi_k
        double np = c->norms.back();
        double nc = frob_norm(bb);
        c->norms.push_back(nc);
        double growth = np > 0.0 ? nc / np : 1.0;
        if (growth > 10.0 && status == 0) {
            status = -3;
            if (fail_k) *fail_k = k;
            return status;
        }
    }
    c->psi = ndeg >= 1 ? bb : a;
    c->hpsi.resize(n);
    apply_h(*c, c->psi.data(), c->hpsi.data(), c->n_bands);
    return status;
}

// Residual-based Chebyshev filter, R-ChFSI (reference_paper/2025 main.tex
// Algorithm 3), for H x = e S x with the approximate inverse D^-1 taken as
// the exact S^-1 (Woodbury), written for the operator S^-1 H on unweighted
// residuals (R~ = D^-1 Z of the paper, which is the same recurrence after the
// similarity D^-1 (.) D):
//   Y   = S^-1 (H X - S X Lam)                     (residual of the Ritz pairs)
//   R_0 = 0, R_1 = (s1/e) Y;  L_0 = 1, L_1 = (s1/e)(Lam - c)
//   R_k = a_k S^-1 H R_{k-1} - a_k c R_{k-1} - s_{k-1} s_k R_{k-2} + a_k Y L_{k-1}
//   L_k = a_k L_{k-1} Lam - a_k c L_{k-1} - s_{k-1} s_k L_{k-2}
//   a_k = 2 s_k / e,  s_1 = e / (lambda_min - c),  s_k = 1 / (2 / s_1 - s_{k-1})
//   X_p = R_p + X L_p
// with the bounds of oracle_spectral_bounds and lambda_min = the lowest Ritz
// value.  In exact arithmetic X_p = C_p(S^-1 H) X / C_p(s_1^-1 ...), the
// sigma-scaled Chebyshev filter of X: the same span as the unscaled filter of
// oracle_chebyshev_filter.  Needs the Ritz values of X (n_eig = n_bands).
int oracle_rchfsi_filter(OracleCtx* c, int ndeg, const double* eig, int n_eig) {
    const int nb = c->n_bands, npw = c->n_pw;
    if (!eig || n_eig != nb || ndeg < 1) return -6;
    double b4[4];
    oracle_spectral_bounds(c, eig, n_eig, b4);
    c->bounds.assign(b4, b4 + 4);
    c->norms.clear();
    const double cc = b4[2], e = b4[3];
    double sigma = e / (eig[0] - cc);
    const double sigma1 = sigma, gamma = 2.0 / sigma1;
    const size_t n = c->psi.size();
    std::vector<cplx> hx(n), sx(n), y(n), t(n), rx(n, 0.0), ry(n), tmp(n);
    apply_h(*c, c->psi.data(), hx.data(), nb);
    apply_s(*c, c->psi.data(), sx.data(), nb);
#pragma omp parallel for
    for (int b = 0; b < nb; ++b)
        for (int g = 0; g < npw; ++g) {
            const size_t i = (size_t)b * npw + g;
            tmp[i] = hx[i] - sx[i] * eig[b];
        }
    apply_sinv(*c, tmp.data(), y.data(), nb);
    std::vector<double> lx(nb, 1.0), ly(nb);
    for (int b = 0; b < nb; ++b) ly[b] = sigma1 / e * (eig[b] - cc);
#pragma omp parallel for
    for (size_t i = 0; i < n; ++i) ry[i] = (sigma1 / e) * y[i];
    for (int k = 2; k <= ndeg; ++k) {
        const double s2 = 1.0 / (gamma - sigma);
        const double a = 2.0 * s2 / e;
        apply_h(*c, ry.data(), tmp.data(), nb);
        apply_sinv(*c, tmp.data(), t.data(), nb);
#pragma omp parallel for
        for (int b = 0; b < nb; ++b)
            for (int g = 0; g < npw; ++g) {
                const size_t i = (size_t)b * npw + g;
                rx[i] = a * t[i] - a * cc * ry[i] - sigma * s2 * rx[i] + a * y[i] * ly[b];
            }
        for (int b = 0; b < nb; ++b) lx[b] = a * ly[b] * eig[b] - a * cc * ly[b] - sigma * s2 * lx[b];
        std::swap(rx, ry);
        std::swap(lx, ly);
        sigma = s2;
    }
#pragma omp parallel for
    for (int b = 0; b < nb; ++b)
        for (int g = 0; g < npw; ++g) {
            const size_t i = (size_t)b * npw + g;
            c->psi[i] = ry[i] + c->psi[i] * ly[b];
        }
    c->hpsi.resize(n);
    apply_h(*c, c->psi.data(), c->hpsi.data(), nb);
    return 0;
}

// Rayleigh-Ritz by Cholesky reduction (subspace_diag.rs:71-391):
// H_sub, S_sub upper triangles + Hermitian fill + symmetrise; S = L L^H;
// B = L^-1 H L^-H (symmetrised); B U = U diag(eps); V = L^-H U;
// psi_new_i = sum_j V_ji psi_j.  Returns 0 or -4 (RayleighRitzFailed).
int oracle_rayleigh_ritz(OracleCtx* c, double* eig_out, int* info) {
    const int nb = c->n_bands, np = c->n_pw;
    std::vector<cplx> H((size_t)nb * nb), S((size_t)nb * nb);
    std::vector<cplx> spsi(c->psi.size());
    apply_s(*c, c->psi.data(), spsi.data(), nb);  // S_sub = psi^H S psi (generalised RR)
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < nb; ++i)
        for (int j = i; j < nb; ++j) {
            const cplx* pi = &c->psi[(size_t)i * np];
            const cplx* pj = &spsi[(size_t)j * np];
            const cplx* hj = &c->hpsi[(size_t)j * np];
            cplx sh = 0.0, ss = 0.0;
            for (int g = 0; g < np; ++g) {
                sh += std::conj(pi[g]) * hj[g];
                ss += std::conj(pi[g]) * pj[g];
            }
            H[(size_t)i * nb + j] = sh; S[(size_t)i * nb + j] = ss;
            if (i != j) { H[(size_t)j * nb + i] = std::conj(sh); S[(size_t)j * nb + i] = std::conj(ss); }
        }
    auto herm = [nb](std::vector<cplx>& m) {
        std::vector<cplx> o = m;
        for (int i = 0; i < nb; ++i)
            for (int j = 0; j < nb; ++j)
                m[(size_t)i * nb + j] = (o[(size_t)i * nb + j] + std::conj(o[(size_t)j * nb + i])) * 0.5;
    };
    herm(H);
    herm(S);
    std::vector<cplx> L = S;
    int inf = cholesky(L, nb);
    if (info) *info = inf;
    if (inf != 0) return -4;
    std::vector<cplx> Li = tri_lower_inverse(L, nb);
    std::vector<cplx> T((size_t)nb * nb, 0.0), B((size_t)nb * nb, 0.0);
    for (int i = 0; i < nb; ++i)
        for (int k = 0; k < nb; ++k) {
            cplx lik = Li[(size_t)i * nb + k];
            if (lik == 0.0) continue;
            for (int j = 0; j < nb; ++j) T[(size_t)i * nb + j] += lik * H[(size_t)k * nb + j];
        }
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            cplx s = 0.0;
            for (int k = 0; k < nb; ++k) s += T[(size_t)i * nb + k] * std::conj(Li[(size_t)j * nb + k]);
            B[(size_t)i * nb + j] = s;
        }
    herm(B);
    std::vector<double> w;
    std::vector<cplx> U;
    jacobi_evd(B, nb, w, U);
    std::vector<cplx> V((size_t)nb * nb, 0.0);  // V = L^-H U
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            cplx s = 0.0;
            for (int k = 0; k < nb; ++k) s += std::conj(Li[(size_t)k * nb + i]) * U[(size_t)k * nb + j];
            V[(size_t)i * nb + j] = s;
        }
    std::vector<cplx> old = c->psi;
#pragma omp parallel for schedule(static)
    for (int g = 0; g < np; ++g)
        for (int i = 0; i < nb; ++i) {
            cplx s = 0.0;
            for (int j = 0; j < nb; ++j) s += V[(size_t)j * nb + i] * old[(size_t)j * np + g];
            c->psi[(size_t)i * np + g] = s;
        }
    c->eig = w;
    if (eig_out) std::memcpy(eig_out, w.data(), sizeof(double) * nb);
    return 0;
}

int oracle_diagonalize(OracleCtx* c, int ndeg, const double* eig, int n_eig, double* eig_out) {
    int fk = 0;
    int st = oracle_chebyshev_filter(c, ndeg, eig, n_eig, &fk);
    if (st) return st;
    int info = 0;
    return oracle_rayleigh_ritz(c, eig_out, &info);
}

// Generalised RR on given arrays: H x = e S x for (h, s) n x n row-major,
// eigenvalues ascending (the cuSOLVER ZHEGVD itype-1 contract of
// src/device/solver.rs:47-95 and the subspace_diag.rs reduction).
int oracle_hegv(int n, const double* h, const double* s, double* w_out, double* v_out) {
    std::vector<cplx> H((size_t)n * n), S((size_t)n * n);
    std::memcpy(H.data(), h, sizeof(cplx) * H.size());
    std::memcpy(S.data(), s, sizeof(cplx) * S.size());
    int inf = cholesky(S, n);
    if (inf) return -4;
    std::vector<cplx> Li = tri_lower_inverse(S, n);
    std::vector<cplx> B((size_t)n * n, 0.0), T((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j) T[(size_t)i * n + j] += Li[(size_t)i * n + k] * H[(size_t)k * n + j];
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            cplx acc = 0.0;
            for (int k = 0; k < n; ++k) acc += T[(size_t)i * n + k] * std::conj(Li[(size_t)j * n + k]);
            B[(size_t)i * n + j] = acc;
        }
    std::vector<double> w;
    std::vector<cplx> U;
    jacobi_evd(B, n, w, U);
    std::memcpy(w_out, w.data(), sizeof(double) * n);
    if (v_out) {
        std::vector<cplx> V((size_t)n * n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                cplx acc = 0.0;
                for (int k = 0; k < n; ++k) acc += std::conj(Li[(size_t)k * n + i]) * U[(size_t)k * n + j];
                V[(size_t)i * n + j] = acc;
            }
        std::memcpy(v_out, V.data(), sizeof(cplx) * V.size());
    }
    return 0;
}

// rho(r) = sum_b f_b |psi_b(r)|^2 / Omega, psi_b(r) = FFT[+1](scatter psi_b)
// (construct_density, src/scf.rs:275-279; design PROJECT_ROOT_PLAN.md:568-611).
void oracle_density(OracleCtx* c, double* rho) {
    const size_t ng = c->ng();
    std::vector<double> acc(ng, 0.0);
#pragma omp parallel
    {
        std::vector<cplx> grid(ng);
        std::vector<double> loc(ng, 0.0);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < c->n_bands; ++b) {
            if (c->occ[b] == 0.0) continue;
            std::fill(grid.begin(), grid.end(), cplx(0.0));
            for (int g = 0; g < c->n_pw; ++g) grid[c->fft_idx[g]] = c->psi[(size_t)b * c->n_pw + g];
            c->fft.run(grid.data(), +1);
            for (size_t r = 0; r < ng; ++r) loc[r] += c->occ[b] * std::norm(grid[r]);
        }
#pragma omp critical
        for (size_t r = 0; r < ng; ++r) acc[r] += loc[r];
    }
    for (size_t r = 0; r < ng; ++r) rho[r] = acc[r] / c->omega;
}

// V_H and V_xc of a density; returns E_H and E_xc; vh, vxc may be null.
static void hartree_xc(OracleCtx* c, const double* rho, double* vh, double* vxc, double* e_h,
                       double* e_xc) {
    const size_t ng = c->ng();
    const double b = 2.0 * M_PI / std::cbrt(c->omega);  // cubic cell
    std::vector<cplx> g(ng);
    for (size_t r = 0; r < ng; ++r) g[r] = rho[r];
    c->fft.run_par(g.data(), -1);
    double eh = 0.0;
    for (int iz = 0; iz < c->nz; ++iz) {
        int l = iz < (c->nz + 1) / 2 ? iz : iz - c->nz;
        for (int iy = 0; iy < c->ny; ++iy) {
            int k = iy < (c->ny + 1) / 2 ? iy : iy - c->ny;
            for (int ix = 0; ix < c->nx; ++ix) {
                int h = ix < (c->nx + 1) / 2 ? ix : ix - c->nx;
                size_t idx = (size_t)ix + (size_t)c->nx * (iy + (size_t)c->ny * iz);
                double g2 = b * b * (double)(h * h + k * k + l * l);
                if (g2 == 0.0) { g[idx] = 0.0; continue; }
                cplx rg = g[idx] / (double)ng;
                eh += 0.5 * c->omega * 4.0 * M_PI * std::norm(rg) / g2;
                g[idx] = 4.0 * M_PI * rg / g2;
            }
        }
    }
    if (vh) {
        c->fft.run_par(g.data(), +1);
        for (size_t r = 0; r < ng; ++r) vh[r] = g[r].real();
    }
    double exc_sum = 0.0;
    for (size_t r = 0; r < ng; ++r) {
        double ex, vx;
        lda_pz(std::max(rho[r], 0.0), ex, vx);
        exc_sum += rho[r] * ex;
        if (vxc) vxc[r] = vx;
    }
    if (e_h) *e_h = eh;
    if (e_xc) *e_xc = exc_sum * c->omega / (double)ng;
}

// V_eff = V_loc + V_H[rho] + V_xc[rho] (build_v_eff, src/scf.rs:157-159).
void oracle_build_veff(OracleCtx* c, const double* rho, double* vh, double* vxc) {
    const size_t ng = c->ng();
    std::vector<double> h(ng), x(ng);
    hartree_xc(c, rho, h.data(), x.data(), nullptr, nullptr);
    for (size_t r = 0; r < ng; ++r) c->veff[r] = c->vloc_r[r] + h[r] + x[r];
    if (vh) std::memcpy(vh, h.data(), sizeof(double) * ng);
    if (vxc) std::memcpy(vxc, x.data(), sizeof(double) * ng);
}

// Pulay / DIIS mixing (DensityHistory::mix, src/mixing.rs:24-27; spec
// plans/phase-2/PHASE_PLAN.md:105-115, 221-230): residuals R_i = out_i - in_i,
// M_ij = <R_i|R_j>, minimise c^T M c with sum c = 1,
// rho_next = sum c_i (in_i + alpha R_i); history capped at max_hist.
void oracle_pulay(OracleCtx* c, const double* rho_in, const double* rho_out, double alpha,
                  int max_hist, double* rho_next) {
    const size_t ng = c->ng();
    std::vector<double> in(rho_in, rho_in + ng), res(ng);
    for (size_t r = 0; r < ng; ++r) res[r] = rho_out[r] - rho_in[r];
    c->hist_rho.push_back(in);
    c->hist_res.push_back(res);
    while ((int)c->hist_rho.size() > max_hist) {
        c->hist_rho.erase(c->hist_rho.begin());
        c->hist_res.erase(c->hist_res.begin());
    }
    const int m = (int)c->hist_rho.size();
    std::vector<double> coef(m, 0.0);
    if (m == 1) coef[0] = 1.0;
    else {
        // bordered system [[M, 1], [1^T, 0]] [c; lam] = [0; 1], Gaussian
        // elimination with partial pivoting
        const int n = m + 1;
        std::vector<double> A((size_t)n * n, 0.0), rhs(n, 0.0);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                double s = 0.0;
                for (size_t r = 0; r < ng; ++r) s += c->hist_res[i][r] * c->hist_res[j][r];
                A[(size_t)i * n + j] = s;
            }
        for (int i = 0; i < m; ++i) { A[(size_t)i * n + m] = 1.0; A[(size_t)m * n + i] = 1.0; }
        rhs[m] = 1.0;
        for (int col = 0; col < n; ++col) {
            int piv = col;
            for (int r = col + 1; r < n; ++r)
                if (std::fabs(A[(size_t)r * n + col]) > std::fabs(A[(size_t)piv * n + col])) piv = r;
            if (piv != col) {
                for (int k = 0; k < n; ++k) std::swap(A[(size_t)col * n + k], A[(size_t)piv * n + k]);
                std::swap(rhs[col], rhs[piv]);
            }
            double d = A[(size_t)col * n + col];
            for (int r = col + 1; r < n; ++r) {
                double f = A[(size_t)r * n + col] / d;
                for (int k = col; k < n; ++k) A[(size_t)r * n + k] -= f * A[(size_t)col * n + k];
                rhs[r] -= f * rhs[col];
            }
        }
        std::vector<double> x(n);
        for (int i = n - 1; i >= 0; --i) {
            double s = rhs[i];
            for (int k = i + 1; k < n; ++k) s -= A[(size_t)i * n + k] * x[k];
            x[i] = s / A[(size_t)i * n + i];
        }
        for (int i = 0; i < m; ++i) coef[i] = x[i];
    }
    for (size_t r = 0; r < ng; ++r) {
        double s = 0.0;
        for (int i = 0; i < m; ++i) s += coef[i] * (c->hist_rho[i][r] + alpha * c->hist_res[i][r]);
        rho_next[r] = s;
    }
}

// Energy of rho_out with band energy from eigenvalues of H[rho_in]:
// E = sum f eps - int (V_H[in] + V_xc[in]) rho_out + E_H[out] + E_xc[out] + E_ewald.
// out5 = {E_total, E_band, E_H[out], E_xc[out], double-counting integral}.
void oracle_energy(OracleCtx* c, const double* rho_in, const double* rho_out, const double* eig,
                   double* out5) {
    const size_t ng = c->ng();
    std::vector<double> vh(ng), vx(ng);
    double eh_in, exc_in, eh, exc;
    hartree_xc(c, rho_in, vh.data(), vx.data(), &eh_in, &exc_in);
    hartree_xc(c, rho_out, nullptr, nullptr, &eh, &exc);
    double dc = 0.0;
    for (size_t r = 0; r < ng; ++r) dc += (vh[r] + vx[r]) * rho_out[r];
    dc *= c->omega / (double)ng;
    double eb = 0.0;
    for (int b = 0; b < c->n_bands; ++b) eb += c->occ[b] * eig[b];
    out5[0] = eb - dc + eh + exc + c->e_ewald;
    out5[1] = eb; out5[2] = eh; out5[3] = exc; out5[4] = dc;
}

// Full SCF (run_scf, src/scf.rs:358-376, with the intended transition
// bodies): V_eff -> diagonalize -> occupations -> density -> energy -> check
// -> Pulay.  The reported energy is the free energy E - kT S.
// The first SCF step runs `first_passes` filter+RR passes from the random
// start.  Returns 0 converged, -1 not converged, or a filter/RR error.
int oracle_scf_run(OracleCtx* c, int ndeg, int max_iter, double tol_per_atom, double alpha,
                   int max_hist, int first_passes, double kT, double* e_hist, int* n_iter,
                   double* eig_out, double* rho_final) {
    const size_t ng = c->ng();
    std::vector<double> rin(ng, 0.0), rout(ng), rnext(ng);
    double nel = 0.0;
    for (double f : c->occ) nel += f;
    for (size_t r = 0; r < ng; ++r) rin[r] = nel / c->omega;
    c->hist_rho.clear();
    c->hist_res.clear();
    std::vector<double> eig;
    double e_prev = 0.0;
    int status = -1;
    int it;
    for (it = 1; it <= max_iter; ++it) {
        oracle_build_veff(c, rin.data(), nullptr, nullptr);
        int passes = it == 1 ? std::max(1, first_passes) : 1;
        std::vector<double> w(c->n_bands);
        for (int p = 0; p < passes; ++p) {
            int st = oracle_diagonalize(c, ndeg, eig.empty() ? nullptr : eig.data(), (int)eig.size(), w.data());
            if (st) { if (n_iter) *n_iter = it; return st; }
            eig = w;
        }
        const double e_ts = fermi_occupations(eig.data(), c->n_bands, nel, kT, c->occ.data());
        oracle_density(c, rout.data());
        double e5[5];
        oracle_energy(c, rin.data(), rout.data(), eig.data(), e5);
        const double etot = e5[0] + e_ts;
        if (e_hist) e_hist[it - 1] = etot;
        if (it > 1 && std::fabs(etot - e_prev) / c->n_atoms_d < tol_per_atom) {
            status = 0;
            e_prev = etot;
            break;
        }
        e_prev = etot;
        oracle_pulay(c, rin.data(), rout.data(), alpha, max_hist, rnext.data());
        rin.swap(rnext);
    }
    if (n_iter) *n_iter = std::min(it, max_iter);
    if (eig_out) std::memcpy(eig_out, eig.data(), sizeof(double) * eig.size());
    if (rho_final) std::memcpy(rho_final, rout.data(), sizeof(double) * ng);
    return status;
}

}  // extern "C"
