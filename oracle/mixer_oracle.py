"""ORACLE — test infrastructure only: CPU restatement of the learned density
mixer (the library's csrc/mixer.cu and its use in chfsi_scf_run).

The mixer has no counterpart in the reference crate (src/mixing.rs:24
DensityHistory::mix is a todo!()); this module states the same arithmetic in
float64 numpy so that the GPU forward pass, gradients, shell features and
targets can be checked against it:

  * MLP 512 -> 256 -> 256 -> 128, GELU (erf form) after the two hidden
    layers, weights rounded to BF16 (round to nearest even) exactly as the
    kernels read them, biases in FP32;
  * loss  L = mean_b sum_s (y_bs - y*_bs)^T M_bs (y_bs - y*_bs) over the
    per-shell pairs (a_s, b_s) with targets (a*, b*, M00, M01, M11);
  * shells  s = min(63, floor(64 sqrt(|G| / 12))), G = 0 excluded;
  * features and least-squares targets from per-shell sums of the G-space
    residual history R_0..R_3, the step D = rho_in - rho_in_prev and the
    error E = rho* - rho_in: per shell, (|R_0|^2, Re<R_0, D>) and for
    t = 1..3 (Re<R_0, R_t>, |R_t|^2), each x 64 / |R_0|^2 and compressed by
    sign(x) log(1 + |x|).

Only tests/ import this module.
"""
import numpy as np
from scipy.special import erf

SHELLS, HIST, N_IN, N_HID, N_OUT, N_T = 64, 4, 512, 256, 128, 5
G_SHELL_MAX = 12.0

OFF_W1 = 0
OFF_B1 = OFF_W1 + N_HID * N_IN
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_OUT * N_HID
N_PARAMS = OFF_B3 + N_OUT


def bf16_round(w):
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(params, quantize=True):
    p = np.asarray(params, dtype=np.float32)
    wq = (bf16_round(p) if quantize else p).astype(np.float64)
    pf = p.astype(np.float64)
    W1 = wq[OFF_W1:OFF_B1].reshape(N_HID, N_IN)
    W2 = wq[OFF_W2:OFF_B2].reshape(N_HID, N_HID)
    W3 = wq[OFF_W3:OFF_B3].reshape(N_OUT, N_HID)
    return W1, pf[OFF_B1:OFF_W2], W2, pf[OFF_B2:OFF_W3], W3, pf[OFF_B3:]


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(params, x, quantize=True):
    W1, b1, W2, b2, W3, b3 = unpack(params, quantize)
    x = np.asarray(x, dtype=np.float32).astype(np.float64).reshape(-1, N_IN)
    z1 = x @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    y = h2 @ W3.T + b3
    return y, (x, z1, h1, z2, h2)


def loss_grad(params, x, t, quantize=True):
    """Loss and gradient w.r.t. the parameter vector (straight through the
    BF16 rounding of the weights; quantize=False drops the rounding, for
    finite-difference checks)."""
    W1, b1, W2, b2, W3, b3 = unpack(params, quantize)
    y, (x, z1, h1, z2, h2) = forward(params, x, quantize)
    B = y.shape[0]
    t = np.asarray(t, dtype=np.float64).reshape(B, SHELLS, N_T)
    ya = y.reshape(B, SHELLS, 2)
    ea = ya[:, :, 0] - t[:, :, 0]
    eb = ya[:, :, 1] - t[:, :, 1]
    m00, m01, m11 = t[:, :, 2], t[:, :, 3], t[:, :, 4]
    loss = np.sum(ea * ea * m00 + 2 * ea * eb * m01 + eb * eb * m11) / B
    dy = np.zeros((B, SHELLS, 2))
    dy[:, :, 0] = 2.0 / B * (m00 * ea + m01 * eb)
    dy[:, :, 1] = 2.0 / B * (m01 * ea + m11 * eb)
    dy = dy.reshape(B, N_OUT)
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = (dy.T @ h2).ravel()
    g[OFF_B3:] = dy.sum(0)
    d2 = (dy @ W3) * gelu_grad(z2)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = (d2 @ W2) * gelu_grad(z1)
    g[OFF_W1:OFF_B1] = (d1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return loss, g


def shell_index(ngrid, recip):
    """Shell of every point of a natural-order numpy FFT grid [nz, ny, nx]
    (255 at G = 0); recip rows are b1, b2, b3 (bohr^-1, 2 pi included)."""
    nx, ny, nz = ngrid
    h = np.fft.fftfreq(nx, 1.0 / nx)
    k = np.fft.fftfreq(ny, 1.0 / ny)
    l = np.fft.fftfreq(nz, 1.0 / nz)
    L, K, H = np.meshgrid(l, k, h, indexing="ij")
    b = np.asarray(recip, dtype=np.float64).reshape(3, 3)
    G = H[..., None] * b[0] + K[..., None] * b[1] + L[..., None] * b[2]
    g = np.sqrt((G * G).sum(-1))
    s = np.minimum(SHELLS - 1, np.floor(SHELLS * np.sqrt(g / G_SHELL_MAX))).astype(np.int64)
    s[(H == 0) & (K == 0) & (L == 0)] = 255
    return s.ravel()


def shell_sums(shell, R, D=None, E=None):
    """Per-shell accumulators (64 x 12) of the library's k_shell_acc; R is a
    list of 1..4 complex G-space arrays (newest first)."""
    acc = np.zeros((SHELLS, 12))
    m = shell != 255
    s = shell[m]

    def add(col, v):
        acc[:, col] += np.bincount(s, weights=v[m], minlength=SHELLS)[:SHELLS]

    r0 = R[0]
    add(0, (np.conj(r0) * r0).real)
    for t in range(1, 4):
        if t < len(R) and R[t] is not None:
            add(t, (np.conj(r0) * R[t]).real)
            add(3 + t, (np.conj(R[t]) * R[t]).real)
    d = np.zeros_like(r0)
    if D is not None:
        d = D
        add(7, (np.conj(d) * d).real)
        add(8, (np.conj(r0) * d).real)
    if E is not None:
        add(9, (np.conj(r0) * E).real)
        add(10, (np.conj(d) * E).real)
        add(11, (np.conj(E) * E).real)
    return acc


def slog(x):
    return np.sign(x) * np.log1p(np.abs(x))


def features_targets(acc):
    """512 features and 64 x 5 targets from the per-shell sums."""
    r2, e2 = acc[:, 0].sum(), acc[:, 11].sum()
    sc = SHELLS / r2 if r2 > 0 else 0.0
    x = np.zeros((SHELLS, HIST, 2))
    x[:, 0, 0] = slog(acc[:, 0] * sc)
    x[:, 0, 1] = slog(acc[:, 8] * sc)
    for h in range(1, HIST):
        x[:, h, 0] = slog(acc[:, h] * sc)
        x[:, h, 1] = slog(acc[:, 3 + h] * sc)
    t = np.zeros((SHELLS, N_T))
    if e2 > 0:
        m00, m01, m11 = acc[:, 0] / e2, acc[:, 8] / e2, acc[:, 7] / e2
        ra, rb = acc[:, 9] / e2, acc[:, 10] / e2
        for s in range(SHELLS):
            ca = cb = 0.0
            if m00[s] > 0:
                if m11[s] <= 1e-12 * m00[s]:
                    ca = ra[s] / m00[s]
                else:
                    lam = 1e-9 * (m00[s] + m11[s])
                    det = (m00[s] + lam) * (m11[s] + lam) - m01[s] ** 2
                    ca = ((m11[s] + lam) * ra[s] - m01[s] * rb[s]) / det
                    cb = ((m00[s] + lam) * rb[s] - m01[s] * ra[s]) / det
            t[s] = [np.clip(ca, -10, 10), np.clip(cb, -10, 10), m00[s], m01[s], m11[s]]
    return x.ravel(), t.ravel()


def trajectory_samples(rho_in, rho_out, rho_star, ngrid, recip):
    """Features and targets of a recorded trajectory (numpy FFTs)."""
    nx, ny, nz = ngrid
    shell = shell_index(ngrid, recip)
    f = lambda r: np.fft.fftn(np.asarray(r).reshape(nz, ny, nx)).ravel()
    T = len(rho_in)
    X = np.zeros((T, N_IN))
    Y = np.zeros((T, SHELLS * N_T))
    hist = []
    star_g = f(rho_star)
    for it in range(T):
        hist.insert(0, f(rho_out[it] - rho_in[it]))
        hist = hist[:HIST]
        D = f(rho_in[it] - rho_in[it - 1]) if it > 0 else None
        E = star_g - f(rho_in[it])
        X[it], Y[it] = features_targets(shell_sums(shell, hist, D, E))
    return X, Y
