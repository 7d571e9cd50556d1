// Host-side dense complex linear algebra for set-up quantities that are
// computed once per run (the Woodbury factor of the ultrasoft overlap).
#include <complex>
#include <cstddef>
#include <utility>
#include <vector>

namespace chfsi {

using zc = std::complex<double>;

// In-place inverse of a dense row-major n x n complex matrix by Gauss-Jordan
// elimination with partial pivoting (rows eliminated in parallel).
bool invert_complex(std::vector<zc>& a, int n) {
    std::vector<zc> inv((size_t)n * n, zc(0.0));
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
        const zc d = 1.0 / a[(size_t)col * n + col];
        for (int k = 0; k < n; ++k) {
            a[(size_t)col * n + k] *= d;
            inv[(size_t)col * n + k] *= d;
        }
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r) {
            if (r == col) continue;
            const zc f = a[(size_t)r * n + col];
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

}  // namespace chfsi
