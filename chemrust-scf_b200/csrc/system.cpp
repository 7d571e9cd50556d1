// Synthetic plane-wave systems: lattice, G-sphere, V_loc(G), Kleinman-Bylander
// projectors beta(G+k), D and q blocks, initial wavefunctions, Ewald energy.
//
// The reference obtains these quantities from chemrust-hamiltonian-core
// (GVectorGrid, compute_beta_g, build_d0_expanded; used at
// src/eigensolver/vnl_data.rs:50-71 and src/scf.rs:5), which is not vendored.
// Here they follow the analytic model of the benchmark systems:
//   V_loc(G)  = -4 pi Z / (Omega G^2) exp(-G^2 rc^2 / 4),  V_loc(0) = 0
//   beta_l(r) = r^l exp(-r^2 / rc^2) Y_lm(r^),  l = 0, 1 (real harmonics)
//   beta_lm(q) = 4 pi / sqrt(Omega) (-i)^l Y_lm(q^) F_l(q) e^{-i q.R},  q = G + k
//   F_l(q)    = int r^2 j_l(q r) r^l e^{-r^2/rc^2} dr
//             = sqrt(pi) / 2^(l+2) rc^(2l+3) q^l exp(-q^2 rc^2 / 4)
// Everything is deterministic in the seed (SplitMix64, one sub-stream per
// purpose; Box-Muller for Gaussian coefficients).
//
// This is set-up code (the reference also builds these on the CPU, once per
// diagonalize: vnl_data.rs:25-89); it is not on the device hot path.
#include "chfsi.h"
#include "system.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace chfsi {

namespace {

constexpr double kPi = 3.14159265358979323846;

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    // uniform in [0, 1)
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    // uniform in (0, 1]
    double uniform_open0() { return 1.0 - uniform(); }
};

// Sub-stream seeds: one independent stream per purpose.
enum Stream : uint64_t { kJitter = 1, kDmat = 2, kQmat = 3, kPsi = 4 };
uint64_t sub_seed(uint64_t seed, Stream st) {
    SplitMix64 m(seed ^ (0xD1B54A32D192ED03ULL * (uint64_t)st));
    return m.next();
}

bool smooth235(int n) {
    if (n <= 0) return false;
    for (int p : {2, 3, 5})
        while (n % p == 0) n /= p;
    return n == 1;
}

int wrap(int h, int n) { return h >= 0 ? h : h + n; }

}  // namespace

int next_smooth235(int n) {
    while (!smooth235(n)) ++n;
    return n;
}

// Ion-ion (point-charge) Ewald energy of a cubic cell with neutralising
// background.
static double ewald_energy(const std::vector<double>& pos, const std::vector<double>& z,
                           double a) {
    const int na = (int)z.size();
    const double omega = a * a * a;
    const double eta = 5.0 / a;
    double e_real = 0.0;
    const int nimg = 2;
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < na; ++j)
            for (int lx = -nimg; lx <= nimg; ++lx)
                for (int ly = -nimg; ly <= nimg; ++ly)
                    for (int lz = -nimg; lz <= nimg; ++lz) {
                        if (i == j && lx == 0 && ly == 0 && lz == 0) continue;
                        double dx = pos[3 * i] - pos[3 * j] + lx * a;
                        double dy = pos[3 * i + 1] - pos[3 * j + 1] + ly * a;
                        double dz = pos[3 * i + 2] - pos[3 * j + 2] + lz * a;
                        double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                        e_real += 0.5 * z[i] * z[j] * std::erfc(eta * r) / r;
                    }
    double e_recip = 0.0;
    const int gm = 10;
    const double b = 2.0 * kPi / a;
    for (int h = -gm; h <= gm; ++h)
        for (int k = -gm; k <= gm; ++k)
            for (int l = -gm; l <= gm; ++l) {
                if (h == 0 && k == 0 && l == 0) continue;
                double gx = b * h, gy = b * k, gz = b * l;
                double g2 = gx * gx + gy * gy + gz * gz;
                double sr = 0.0, si = 0.0;
                for (int i = 0; i < na; ++i) {
                    double ph = gx * pos[3 * i] + gy * pos[3 * i + 1] + gz * pos[3 * i + 2];
                    sr += z[i] * std::cos(ph);
                    si += z[i] * std::sin(ph);
                }
                e_recip += (2.0 * kPi / omega) * (sr * sr + si * si) *
                           std::exp(-g2 / (4.0 * eta * eta)) / g2;
            }
    double zsum = 0.0, z2 = 0.0;
    for (double zi : z) { zsum += zi; z2 += zi * zi; }
    double e_self = -eta / std::sqrt(kPi) * z2;
    double e_bg = -kPi * zsum * zsum / (2.0 * omega * eta * eta);
    return e_real + e_recip + e_self + e_bg;
}

chfsi_status generate_system(const chfsi_synth_params& p, System& s, const double* pos_override) {
    if (p.n_rep < 1 || p.a_conv <= 0 || p.ecut <= 0 || p.lmax < 0 || p.lmax > 1 ||
        p.n_shell < 0 || p.n_shell > 4)
        return CHFSI_ERR_BAD_INPUT;
    s.params = p;
    const double a = p.a_conv * p.n_rep;
    s.a = a;
    s.omega = a * a * a;
    std::memset(s.lattice, 0, sizeof(s.lattice));
    s.lattice[0] = s.lattice[4] = s.lattice[8] = a;

    // ---- atoms ----
    std::vector<std::array<double, 3>> basis;
    switch (p.lattice) {
    case CHFSI_LATTICE_DIAMOND: {
        const double fcc[4][3] = {{0, 0, 0}, {0, .5, .5}, {.5, 0, .5}, {.5, .5, 0}};
        for (int i = 0; i < 4; ++i) basis.push_back({fcc[i][0], fcc[i][1], fcc[i][2]});
        for (int i = 0; i < 4; ++i)
            basis.push_back({fcc[i][0] + .25, fcc[i][1] + .25, fcc[i][2] + .25});
        break;
    }
    case CHFSI_LATTICE_SC: basis.push_back({0, 0, 0}); break;
    case CHFSI_LATTICE_BCC:
        basis.push_back({0, 0, 0});
        basis.push_back({.5, .5, .5});
        break;
    default: return CHFSI_ERR_BAD_INPUT;
    }
    SplitMix64 rj(sub_seed(p.seed, kJitter));
    s.pos.clear();
    s.zion.clear();
    for (int i = 0; i < p.n_rep; ++i)
        for (int j = 0; j < p.n_rep; ++j)
            for (int k = 0; k < p.n_rep; ++k)
                for (auto& bf : basis) {
                    const double c[3] = {(i + bf[0]) * p.a_conv, (j + bf[1]) * p.a_conv,
                                         (k + bf[2]) * p.a_conv};
                    for (int d = 0; d < 3; ++d)
                        s.pos.push_back(c[d] + (2.0 * rj.uniform() - 1.0) * p.jitter);
                    s.zion.push_back(p.z_val);
                }
    s.n_atoms = (int)s.zion.size();
    if (pos_override) std::memcpy(s.pos.data(), pos_override, sizeof(double) * s.pos.size());
    s.n_elec = p.z_val * s.n_atoms;
    s.n_occ = (int)std::ceil(s.n_elec / 2.0 - 1e-9);
    s.n_bands = p.n_bands > 0 ? p.n_bands : (int)std::ceil(1.25 * s.n_occ - 1e-9);
    if (s.n_bands < s.n_occ) return CHFSI_ERR_BAD_INPUT;
    s.occ.assign(s.n_bands, 0.0);
    {
        double left = s.n_elec;
        for (int b = 0; b < s.n_bands && left > 0; ++b) {
            s.occ[b] = std::min(2.0, left);
            left -= s.occ[b];
        }
    }

    // ---- plane-wave sphere: 1/2 |G+k|^2 <= ecut ----
    const double bvec = 2.0 * kPi / a;
    const double g2cut = 2.0 * p.ecut;
    const double kc[3] = {p.kpt[0] * bvec, p.kpt[1] * bvec, p.kpt[2] * bvec};
    const int mm = (int)std::floor(std::sqrt(g2cut) / bvec) + 2;
    struct PW { int h, k, l; double g2; };
    std::vector<PW> pws;
    int mabs[3] = {0, 0, 0};
    for (int h = -mm; h <= mm; ++h)
        for (int k = -mm; k <= mm; ++k)
            for (int l = -mm; l <= mm; ++l) {
                double gx = h * bvec + kc[0], gy = k * bvec + kc[1], gz = l * bvec + kc[2];
                double g2 = gx * gx + gy * gy + gz * gz;
                if (g2 <= g2cut) {
                    pws.push_back({h, k, l, g2});
                    mabs[0] = std::max(mabs[0], std::abs(h));
                    mabs[1] = std::max(mabs[1], std::abs(k));
                    mabs[2] = std::max(mabs[2], std::abs(l));
                }
            }
    for (int d = 0; d < 3; ++d) {
        int n = p.ngrid[d] > 0 ? p.ngrid[d] : next_smooth235(4 * mabs[d] + 1);
        if (n < 2 * mabs[d] + 1) return CHFSI_ERR_BAD_INPUT;
        s.ngrid[d] = n;
        const int nd = p.ngrid_density[d] > 0 ? p.ngrid_density[d] : n;
        if (nd < n) return CHFSI_ERR_BAD_INPUT;
        s.ngrid_density[d] = nd;
    }
    s.uspp = p.uspp;
    s.q_width = p.q_width;
    const int nx = s.ngrid[0], ny = s.ngrid[1], nz = s.ngrid[2];
    // Sort by column (iy, ix) wrapped, then l ascending: every (x,y) column
    // owns one contiguous run of plane waves.
    std::sort(pws.begin(), pws.end(), [&](const PW& u, const PW& v) {
        int cu = wrap(u.k, ny) * nx + wrap(u.h, nx);
        int cv = wrap(v.k, ny) * nx + wrap(v.h, nx);
        if (cu != cv) return cu < cv;
        return u.l < v.l;
    });
    s.n_pw = (int)pws.size();
    s.miller.resize(3 * (size_t)s.n_pw);
    s.kinetic.resize(s.n_pw);
    double g2max = 0.0;
    for (int g = 0; g < s.n_pw; ++g) {
        s.miller[3 * g] = pws[g].h;
        s.miller[3 * g + 1] = pws[g].k;
        s.miller[3 * g + 2] = pws[g].l;
        s.kinetic[g] = 0.5 * pws[g].g2;
        g2max = std::max(g2max, pws[g].g2);
    }
    s.gmax = std::sqrt(g2max);
    {
        int ncol = 0, last = -1;
        for (auto& q : pws) {
            int c = wrap(q.k, ny) * nx + wrap(q.h, nx);
            if (c != last) { ++ncol; last = c; }
        }
        s.n_columns = ncol;
    }

    // ---- V_loc(G) S(G) on the full grid (Nyquist planes zeroed) ----
    const size_t ng = (size_t)nx * ny * nz;
    s.vloc_g.assign(2 * ng, 0.0);
    {
        const int na = s.n_atoms;
        std::vector<double> fr(3 * (size_t)na);
        for (int i = 0; i < 3 * na; ++i) fr[i] = s.pos[i] / a;
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < nz; ++iz) {
            int l = iz < (nz + 1) / 2 ? iz : iz - nz;
            for (int iy = 0; iy < ny; ++iy) {
                int k = iy < (ny + 1) / 2 ? iy : iy - ny;
                for (int ix = 0; ix < nx; ++ix) {
                    int h = ix < (nx + 1) / 2 ? ix : ix - nx;
                    size_t idx = (size_t)ix + (size_t)nx * (iy + (size_t)ny * iz);
                    if ((h == 0 && k == 0 && l == 0) || (nx % 2 == 0 && 2 * std::abs(h) == nx) ||
                        (ny % 2 == 0 && 2 * std::abs(k) == ny) ||
                        (nz % 2 == 0 && 2 * std::abs(l) == nz))
                        continue;
                    double gx = h * bvec, gy = k * bvec, gz = l * bvec;
                    double g2 = gx * gx + gy * gy + gz * gz;
                    double v = -4.0 * kPi * p.z_val / (s.omega * g2) *
                               std::exp(-g2 * p.rc_loc * p.rc_loc / 4.0);
                    double sr = 0.0, si = 0.0;
                    for (int i = 0; i < na; ++i) {
                        double ph = -2.0 * kPi *
                                    (h * fr[3 * i] + k * fr[3 * i + 1] + l * fr[3 * i + 2]);
                        sr += std::cos(ph);
                        si += std::sin(ph);
                    }
                    s.vloc_g[2 * idx] = v * sr;
                    s.vloc_g[2 * idx + 1] = v * si;
                }
            }
        }
    }

    // ---- projectors ----
    const int n_lm = (p.lmax + 1) * (p.lmax + 1);
    const int ne = p.n_shell * n_lm;
    s.n_proj = ne * s.n_atoms;
    s.n_ions_proj = ne > 0 ? s.n_atoms : 0;
    s.proj_offsets.assign(s.n_ions_proj + 1, 0);
    for (int i = 0; i <= s.n_ions_proj; ++i) s.proj_offsets[i] = i * ne;
    s.beta.assign(2 * (size_t)s.n_proj * s.n_pw, 0.0);
    s.dmat.assign(2 * (size_t)s.n_ions_proj * ne * ne, 0.0);
    s.qmat.assign(2 * (size_t)s.n_ions_proj * ne * ne, 0.0);
    if (ne > 0) {
        const double pref = 4.0 * kPi / std::sqrt(s.omega);
        const double y00 = 1.0 / std::sqrt(4.0 * kPi);
        const double y1 = std::sqrt(3.0 / (4.0 * kPi));
#pragma omp parallel for schedule(dynamic, 1)
        for (int ia = 0; ia < s.n_atoms; ++ia) {
            const double* R = &s.pos[3 * ia];
            for (int g = 0; g < s.n_pw; ++g) {
                double qx = pws[g].h * bvec + kc[0], qy = pws[g].k * bvec + kc[1],
                       qz = pws[g].l * bvec + kc[2];
                double q2 = qx * qx + qy * qy + qz * qz;
                double ph = -(qx * R[0] + qy * R[1] + qz * R[2]);
                double cr = std::cos(ph), ci = std::sin(ph);
                for (int sh = 0; sh < p.n_shell; ++sh) {
                    double rc = p.rc_proj[sh];
                    double e = std::exp(-q2 * rc * rc / 4.0);
                    int base = ia * ne + sh * n_lm;
                    // l = 0: real radial factor times phase
                    double f0 = pref * y00 * (std::sqrt(kPi) / 4.0) * rc * rc * rc * e;
                    size_t o = 2 * ((size_t)base * s.n_pw + g);
                    s.beta[o] = f0 * cr;
                    s.beta[o + 1] = f0 * ci;
                    if (p.lmax >= 1) {
                        // l = 1: (-i) sqrt(3/4pi) (sqrt(pi)/8) rc^5 q_m e
                        double f1 = pref * y1 * (std::sqrt(kPi) / 8.0) * std::pow(rc, 5) * e;
                        const double qm[3] = {qx, qy, qz};
                        for (int m = 0; m < 3; ++m) {
                            double amp = f1 * qm[m];
                            // (-i) * amp * (cr + i ci) = amp*ci - i amp*cr
                            size_t o1 = 2 * ((size_t)(base + 1 + m) * s.n_pw + g);
                            s.beta[o1] = amp * ci;
                            s.beta[o1 + 1] = -amp * cr;
                        }
                    }
                }
            }
        }
        SplitMix64 rd(sub_seed(p.seed, kDmat));
        SplitMix64 rq(sub_seed(p.seed, kQmat));
        for (int ia = 0; ia < s.n_atoms; ++ia) {
            double* D = &s.dmat[2 * (size_t)ia * ne * ne];
            for (int sh = 0; sh < p.n_shell; ++sh)
                for (int l = 0; l <= p.lmax; ++l) {
                    double d = p.d_min + (p.d_max - p.d_min) * rd.uniform();
                    int first = sh * n_lm + (l == 0 ? 0 : 1);
                    int cnt = l == 0 ? 1 : 3;
                    for (int m = 0; m < cnt; ++m) D[2 * ((first + m) * ne + (first + m))] = d;
                }
            if (p.uspp) {
                // q couples the shells of one (l, m) channel: per l a symmetric
                // n_shell x n_shell block with entries U[-q_amp, q_amp].
                double* Q = &s.qmat[2 * (size_t)ia * ne * ne];
                for (int l = 0; l <= p.lmax; ++l)
                    for (int s1 = 0; s1 < p.n_shell; ++s1)
                        for (int s2 = s1; s2 < p.n_shell; ++s2) {
                            double qv = p.q_amp * (2.0 * rq.uniform() - 1.0);
                            int cnt = l == 0 ? 1 : 3;
                            for (int m = 0; m < cnt; ++m) {
                                int i1 = s1 * n_lm + (l == 0 ? 0 : 1 + m);
                                int i2 = s2 * n_lm + (l == 0 ? 0 : 1 + m);
                                Q[2 * (i1 * ne + i2)] = qv;
                                Q[2 * (i2 * ne + i1)] = qv;
                            }
                        }
            }
        }
    }

    // ---- initial wavefunctions: complex Gaussian (Box-Muller) ----
    s.psi0.resize(2 * (size_t)s.n_bands * s.n_pw);
    {
        SplitMix64 rp(sub_seed(p.seed, kPsi));
        for (size_t i = 0; i < (size_t)s.n_bands * s.n_pw; ++i) {
            double u1 = rp.uniform_open0(), u2 = rp.uniform();
            double r = std::sqrt(-2.0 * std::log(u1));
            s.psi0[2 * i] = r * std::cos(2.0 * kPi * u2);
            s.psi0[2 * i + 1] = r * std::sin(2.0 * kPi * u2);
        }
    }

    s.e_ewald = ewald_energy(s.pos, s.zion, a);
    return CHFSI_OK;
}

}  // namespace chfsi

// ------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------
using chfsi::System;

struct chfsi_system : System {};

extern "C" {

chfsi_status chfsi_synth_defaults(int cfg, chfsi_synth_params* p) {
    if (!p) return CHFSI_ERR_BAD_INPUT;
    std::memset(p, 0, sizeof(*p));
    p->lattice = CHFSI_LATTICE_DIAMOND;
    p->a_conv = 10.26;
    p->jitter = 0.05;
    p->z_val = 4.0;
    p->rc_loc = 1.0;
    p->seed = 0;
    switch (cfg) {
    case 0:  // 8 atoms, local only, Ecut 15, 40^3, 20 bands
        p->n_rep = 1; p->ecut = 15.0;
        p->ngrid[0] = p->ngrid[1] = p->ngrid[2] = 40;
        p->n_bands = 20;
        break;
    case 1:  // 64 atoms, KB l=0,1 rc 1.2, Ecut 20, 72^3, 160 bands
        p->n_rep = 2; p->ecut = 20.0;
        p->ngrid[0] = p->ngrid[1] = p->ngrid[2] = 72;
        p->n_bands = 160;
        p->n_shell = 1; p->rc_proj[0] = 1.2; p->lmax = 1;
        p->d_min = 0.5; p->d_max = 2.0;
        break;
    case 2:  // 216 atoms, 2 shells x (l=0,1), q_ij, Ecut 25, 108^3, 576 bands
        p->n_rep = 3; p->ecut = 25.0;
        p->ngrid[0] = p->ngrid[1] = p->ngrid[2] = 108;
        p->n_bands = 576;
        p->n_shell = 2; p->rc_proj[0] = 1.0; p->rc_proj[1] = 1.4; p->lmax = 1;
        p->d_min = 0.5; p->d_max = 2.0;
        p->uspp = 1; p->q_width = 0.8; p->q_amp = 0.1;
        p->ngrid_density[0] = p->ngrid_density[1] = p->ngrid_density[2] = 144;
        break;
    default: return CHFSI_ERR_BAD_INPUT;
    }
    return CHFSI_OK;
}

chfsi_status chfsi_system_generate(const chfsi_synth_params* p, chfsi_system** out) {
    if (!p || !out) return CHFSI_ERR_BAD_INPUT;
    *out = nullptr;
    chfsi_system* s = new (std::nothrow) chfsi_system();
    if (!s) return CHFSI_ERR_OUT_OF_MEMORY;
    chfsi_status st;
    try {
        st = chfsi::generate_system(*p, *s);
    } catch (const std::bad_alloc&) {
        st = CHFSI_ERR_OUT_OF_MEMORY;
    }
    if (st != CHFSI_OK) { delete s; return st; }
    *out = s;
    return CHFSI_OK;
}

chfsi_status chfsi_system_generate_at(const chfsi_synth_params* p, const double* positions,
                                      chfsi_system** out) {
    if (!p || !out || !positions) return CHFSI_ERR_BAD_INPUT;
    *out = nullptr;
    chfsi_system* s = new (std::nothrow) chfsi_system();
    if (!s) return CHFSI_ERR_OUT_OF_MEMORY;
    chfsi_status st;
    try {
        st = chfsi::generate_system(*p, *s, positions);
    } catch (const std::bad_alloc&) {
        st = CHFSI_ERR_OUT_OF_MEMORY;
    }
    if (st != CHFSI_OK) { delete s; return st; }
    *out = s;
    return CHFSI_OK;
}

void chfsi_system_destroy(chfsi_system* s) { delete s; }

chfsi_status chfsi_system_get_info(const chfsi_system* s, chfsi_system_info* o) {
    if (!s || !o) return CHFSI_ERR_BAD_INPUT;
    std::memset(o, 0, sizeof(*o));
    for (int d = 0; d < 3; ++d) o->ngrid[d] = s->ngrid[d];
    for (int d = 0; d < 3; ++d) o->ngrid_density[d] = s->ngrid_density[d];
    o->q_width = s->q_width;
    o->uspp = s->uspp;
    o->n_pw = s->n_pw;
    o->n_bands = s->n_bands;
    o->n_occ = s->n_occ;
    o->n_atoms = s->n_atoms;
    o->n_proj = s->n_proj;
    o->n_ions_with_proj = s->n_ions_proj;
    o->n_columns = s->n_columns;
    o->omega = s->omega;
    o->n_elec = s->n_elec;
    o->gmax = s->gmax;
    o->e_ewald = s->e_ewald;
    std::memcpy(o->lattice, s->lattice, sizeof(o->lattice));
    return CHFSI_OK;
}

#define CHFSI_COPY_OUT(field, T)                                                    \
    if (!s || !out) return CHFSI_ERR_BAD_INPUT;                                     \
    std::memcpy(out, s->field.data(), s->field.size() * sizeof(s->field[0]));       \
    return CHFSI_OK;

chfsi_status chfsi_system_get_miller(const chfsi_system* s, int32_t* out) { CHFSI_COPY_OUT(miller, int32_t) }
chfsi_status chfsi_system_get_kinetic(const chfsi_system* s, double* out) { CHFSI_COPY_OUT(kinetic, double) }
chfsi_status chfsi_system_get_vloc_g(const chfsi_system* s, chfsi_c128* out) { CHFSI_COPY_OUT(vloc_g, double) }
chfsi_status chfsi_system_get_beta(const chfsi_system* s, chfsi_c128* out) { CHFSI_COPY_OUT(beta, double) }
chfsi_status chfsi_system_get_proj_offsets(const chfsi_system* s, int32_t* out) { CHFSI_COPY_OUT(proj_offsets, int32_t) }
chfsi_status chfsi_system_get_dmat(const chfsi_system* s, chfsi_c128* out) { CHFSI_COPY_OUT(dmat, double) }
chfsi_status chfsi_system_get_qmat(const chfsi_system* s, chfsi_c128* out) { CHFSI_COPY_OUT(qmat, double) }
chfsi_status chfsi_system_get_psi0(const chfsi_system* s, chfsi_c128* out) { CHFSI_COPY_OUT(psi0, double) }
chfsi_status chfsi_system_get_occupations(const chfsi_system* s, double* out) { CHFSI_COPY_OUT(occ, double) }
chfsi_status chfsi_system_get_positions(const chfsi_system* s, double* out) { CHFSI_COPY_OUT(pos, double) }

}  // extern "C"
