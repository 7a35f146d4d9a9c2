"""The index arithmetic of the shared-memory lane stage of the 512-point line
transform (qp_line.cuh, reg_line_tail_xs), restated in numpy on the CPU.

The kernel splits the 32-point DFT over the lanes as 8 x 4 (lane l = q + 4 b):
lane t = 4 r + q gathers f_r(q + 4 b) from an XOR-swizzled exchange buffer,
runs an 8-point DFT, a twiddle exp(-2 pi i q c / 32) and a 4-point DFT over q
across four lanes (radix-2, xor 2 then xor 1), and leaves Z[r + 8 (c + 8
brev2(q))] in register c; a second swizzled exchange hands lane l its block
Z[8 l + k2] and the partners Z[256 - 8 l - k2] of the real-FFT unscramble.
This test replays those formulas exactly as written in the kernel and checks
them against numpy's FFT and against the DST-I / DCT-I definitions, and that
both exchanges are bijections whose accesses are free of bank conflicts."""
import numpy as np

P = 8
N = 64 * P
H = N // 2


def brev2(q):
    return ((q & 1) << 1) | (q >> 1)


def W(n, e):
    return np.exp(-2j * np.pi * e / n)


def dft8(x):
    """The kernel's dft8 (radix 2 x 4, natural order in and out)."""
    r = np.sqrt(0.5)
    a0, a1 = x[0] + x[4], x[0] - x[4]
    b0, b1 = x[2] + x[6], x[2] - x[6]
    c0, c1 = x[1] + x[5], x[1] - x[5]
    d0, d1 = x[3] + x[7], x[3] - x[7]
    e0, e1, g0, g1 = a0 + b0, a0 - b0, c0 + d0, c0 - d0
    bb = complex(b1.imag, -b1.real)
    cc = complex(r * (c1.real + c1.imag), r * (c1.imag - c1.real))
    dd = complex(r * (d1.imag - d1.real), -r * (d1.real + d1.imag))
    h0, h1, k0, k1 = a1 + bb, a1 - bb, cc + dd, cc - dd
    out = [0j] * 8
    out[0], out[4] = e0 + g0, e0 - g0
    out[2] = complex(e1.real + g1.imag, e1.imag - g1.real)
    out[6] = complex(e1.real - g1.imag, e1.imag + g1.real)
    out[1], out[5] = h0 + k0, h0 - k0
    out[3] = complex(h1.real + k1.imag, h1.imag - k1.real)
    out[7] = complex(h1.real - k1.imag, h1.imag + k1.real)
    return out


def lane_stage(z):
    """Steps 3-6 of the kernel for the complex sequence z (length H): returns
    (A, B) with A[l][k2] = Z[8 l + k2] and B[l][k2] the unscramble partner as
    the kernel reads them, plus the two exchange buffers' index lists."""
    # lane l holds z[l + 32 a]; P-point DFT over a and the twiddle
    w = np.array([[sum(z[l + 32 * a] * W(P, a * k2) for a in range(P)) * W(H, l * k2)
                   for k2 in range(P)] for l in range(32)])
    X = {}
    idx1 = []
    for l in range(32):
        for k2 in range(P):
            i = 32 * k2 + (l ^ (4 * (k2 & 3)))
            idx1.append((k2, l, i))
            X[i] = w[l][k2]
    f = np.zeros((32, 8), complex)
    for t in range(32):
        r, q = t >> 2, t & 3
        g = dft8([X[32 * r + ((q + 4 * b) ^ (4 * (r & 3)))] for b in range(8)])
        f[t] = [g[c] * W(32, q * c) for c in range(8)]
    # 4-point DFT over q across lanes: radix 2, xor 2 (times -i on q = 3), xor 1
    for s in (2, 1):
        nf = f.copy()
        for t in range(32):
            q = t & 3
            p = f[t ^ s]
            if q & s:
                d = p - f[t]
                nf[t] = d * (-1j) if (s == 2 and q == 3) else d
            else:
                nf[t] = f[t] + p
        f = nf
    Y = {}
    idx2 = []
    for t in range(32):
        r, q = t >> 2, t & 3
        for c in range(8):
            kap = c + 8 * brev2(q)
            i = 8 * kap + (r ^ ((kap >> 1) & 7))
            idx2.append((t, c, i))
            Y[i] = f[t][c]
    A = np.zeros((32, P), complex)
    B = np.zeros((32, P), complex)
    for l in range(32):
        sw = (l >> 1) & 7
        lp, swp, l0 = 31 - l, ((31 - l) >> 1) & 7, (32 - l) & 31
        for k2 in range(P):
            A[l][k2] = Y[8 * l + (k2 ^ sw)]
            B[l][k2] = Y[8 * lp + ((8 - k2) ^ swp)] if k2 else Y[8 * l0 + ((l0 >> 1) & 7)]
    return A, B, idx1, idx2


def test_lane_stage_gives_the_fft_blocks_and_partners():
    rng = np.random.default_rng(4)
    z = rng.standard_normal(H) + 1j * rng.standard_normal(H)
    A, B, _, _ = lane_stage(z)
    Z = np.fft.fft(z)
    for l in range(32):
        for k2 in range(P):
            k = k2 + P * l
            assert abs(A[l][k2] - Z[k]) < 1e-9 * np.abs(Z).max()
            if k:
                assert abs(B[l][k2] - Z[H - k]) < 1e-9 * np.abs(Z).max()


def test_exchanges_are_bijections_without_bank_conflicts():
    _, _, idx1, idx2 = lane_stage(np.zeros(H, complex))
    assert sorted(i for _, _, i in idx1) == list(range(32 * P))
    assert sorted(i for _, _, i in idx2) == list(range(32 * P))
    # 8-byte accesses: a half warp touches 16 distinct 8-byte bank pairs
    # (index mod 16) when it is conflict free
    for k2 in range(P):  # first exchange, stores (one per k2)
        for h in (0, 16):
            pairs = {(32 * k2 + (l ^ (4 * (k2 & 3)))) % 16 for l in range(h, h + 16)}
            assert len(pairs) == 16
    for b in range(8):  # first exchange, strided loads (one per b)
        for h in (0, 16):
            pairs = set()
            for t in range(h, h + 16):
                r, q = t >> 2, t & 3
                pairs.add((32 * r + ((q + 4 * b) ^ (4 * (r & 3)))) % 16)
            assert len(pairs) == 16
    for k2 in range(P):  # second exchange, block loads (one per k2)
        for h in (0, 16):
            pairs = {(8 * l + (k2 ^ ((l >> 1) & 7))) % 16 for l in range(h, h + 16)}
            assert len(pairs) == 16


def test_line_transform_matches_sine_and_cosine_definitions():
    """The whole line (pre-twiddle, lane stage, unscramble, prefix sum) with
    the kernel's block order, against the DST-I / DCT-I sums."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal(N + 1)
    jj = np.arange(1, N)
    sn = np.sin(np.pi * np.arange(N + 1) / N)
    cs = np.cos(np.pi * np.arange(N + 1) / N)
    for parity in (0, 1):
        y = np.zeros(N)
        for j in range(N):
            a, b = x[j], (x[N - j] if j else x[N])
            if parity == 0:
                y[j] = 0.0 if j == 0 else sn[j] * (a + b) + 0.5 * (a - b)
            else:
                y[j] = 0.5 * (a + b) - sn[j] * (a - b)
        sigma = 0.5 * (x[0] - x[N]) + np.sum(x[1:N] * cs[1:N]) if parity else 0.0
        A, B, _, _ = lane_stage(y[0::2] + 1j * y[1::2])
        out = np.zeros(N + 1)
        runs, evs, ods = [], [], []
        yh = 0.0
        for l in range(32):
            run, ev, od = 0.0, [], []
            for k2 in range(P):
                k = k2 + P * l
                a, b = A[l][k2], np.conj(B[l][k2])
                if k == 0:
                    Y = complex(a.real + a.imag, 0.0)
                    yh = a.real - a.imag
                else:
                    E, D = 0.5 * (a + b), a - b
                    u = W(N, k) * D
                    Y = complex(E.real + 0.5 * u.imag, E.imag - 0.5 * u.real)
                if parity == 0:
                    ev.append(0.0 if k == 0 else -2 * Y.imag)
                    run += Y.real if k == 0 else 2 * Y.real
                else:
                    ev.append(2 * Y.real)
                    run += 0.0 if k == 0 else -2 * Y.imag
                od.append(run)
            runs.append(run)
            evs.append(ev)
            ods.append(od)
        inc = np.cumsum(runs)
        for l in range(32):
            base = inc[l] - runs[l] + (2 * sigma if parity else 0.0)
            for k2 in range(P):
                k = k2 + P * l
                out[2 * k], out[2 * k + 1] = evs[l][k2], base + ods[l][k2]
        out[N] = 2 * yh if parity else 0.0
        m = np.arange(N + 1)
        if parity == 0:
            ref = np.array([2 * np.sum(x[1:N] * np.sin(np.pi * jj * mm / N)) for mm in m])
        else:
            ref = np.array([x[0] + (-1) ** mm * x[N] + 2 * np.sum(x[1:N] * np.cos(np.pi * jj * mm / N))
                            for mm in m])
        assert np.abs(out - ref).max() < 1e-10 * np.abs(ref).max(), parity
