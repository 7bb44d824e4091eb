"""CPU model of the packed MSV pre-screen (csrc/prescreen.cuh), the checker of
its integer arithmetic: the bound the kernel computes for one (profile,
target) pair, bit for bit.

The pre-screen has no counterpart in the reference (its MSV, src/hmmer/dp.rs:92-145,
is f32 only); what the tests require of it is (1) the kernel computes exactly
this model, and (2) the model's bound is never below the reference's f32 MSV
score, so no pair the reference passes through F1 is dropped.
"""
import ctypes
import math

import numpy as np

Q16 = 512                # cells: units of 2^-9 nat
Q32 = 1 << 20            # specials: units of 2^-20 nat
RHO32 = 8                # 2^-17 nat in units of 2^-20
EFLOOR, EPAD, BEFLOOR = -8192, -16384, -16384
NEG16, NEG32 = -32768, -(1 << 30)
LN2_F32 = np.float32(0.693147182464599609375)

_libm = ctypes.CDLL("libm.so.6")
_libm.logf.restype = ctypes.c_float
_libm.logf.argtypes = [ctypes.c_float]


def quantize(msc, m):
    """Rounded-up int16 scores of columns 1..m (25 rows) and the profile's cap."""
    e = np.asarray(msc, np.float32)[:, 1:m + 1]
    finite = e > np.float32(-1e30)
    u = np.full(e.shape, EFLOOR, np.int64)
    u[finite] = np.maximum(np.ceil((e[finite].astype(np.float64) + 2.0 ** -12) * Q16), EFLOOR).astype(np.int64)
    emax = max(EFLOOR, int(u[finite].max())) if finite.any() else EFLOOR
    return u, 32767 - emax, emax


def _q32_up(x):
    """f32 constant x in units of 2^-20 nat, rounded up, plus rho (the device's q32_up)."""
    return int(math.ceil(float(np.float32(x)) * Q32)) + RHO32


def _f32_round_up(v):
    f = np.float32(v)
    if float(f) < v:
        f = np.nextafter(f, np.float32(np.inf))
    return f


def msv_bound(msc, m, msv_tbm, width, dsq):
    """The pre-screen's bound (f32 nats) for one pair; inf when a row maximum
    exceeded the cap; NaN for an empty target.  `width` = G * C of the
    profile's MSV shape (columns past m are padding with score -32 nats)."""
    L = len(dsq)
    if L == 0:
        return np.float32(np.nan)
    u, cap, emax = quantize(msc, m)
    if emax >= 8192:
        return np.float32(np.nan)
    e = np.full((25, width), EPAD, np.int64)
    e[:, :m] = u
    lf = np.float32(L)
    tloop = _libm.logf(np.float32(lf / (lf + np.float32(3.0))))
    tmove = _libm.logf(np.float32(np.float32(3.0) / (lf + np.float32(3.0))))
    tl, tm = _q32_up(tloop), _q32_up(tmove)
    q_tbm = int(math.ceil((float(np.float32(msv_tbm)) + 2.0 ** -17) * Q32))
    nln2 = int(math.ceil(float(-LN2_F32) * Q32)) + RHO32
    prev = np.full(width, NEG16, np.int64)
    xn, xj = 0, NEG32
    be = max((tm + q_tbm + 2047) >> 11, BEFLOOR)
    for x in dsq:
        shifted = np.empty(width, np.int64)
        shifted[0] = NEG16
        shifted[1:] = prev[:-1]
        cur = e[int(x)] + np.maximum(shifted, be)
        xe = int(cur.max())
        if xe > cap:
            return np.float32(np.inf)
        xj = max(xj + tl, xe * 2048 + nln2)
        xn += tl
        xb = max(xn, xj) + tm
        be = max((xb + q_tbm + 2047) >> 11, BEFLOOR)
        prev = cur
    return np.float32(_f32_round_up(xj + tm) * np.float32(2.0 ** -20))


# ---- packed Viterbi pre-screen (csrc/prescreen.cuh vit16_kernel) ----------
# The kernel's cells are int16 in units of 2^-9 nat; its lanes hold columns in
# chunks, but the lazy D-chain carry converges to the sequential recurrence
# (the provisional carry is below every D value), so the model needs only the
# width G*C of the profile's pre-screen shape.
V_TFLOOR, V_BMFLOOR, V_EFLOOR, V_BFLOOR = -4096, -8192, -4096, -4096
V_INIT = -16384
VIT16_WIDTHS = (32, 64, 128, 256, 512)   # kVit16Shapes: (4,8) (8,8) (16,8) (32,8) (32,16)
# transition rows of the oracle's t8 (mm mi md im ii dm dd bm)
_TMM, _TMI, _TMD, _TIM, _TII, _TDM, _TDD, _TBM = range(8)

_libm.log.restype = ctypes.c_double
_libm.log.argtypes = [ctypes.c_double]


def vit16_width(m):
    """Width G*C of the pre-screen shape of a profile of M nodes (None: not pre-screened)."""
    return next((w for w in VIT16_WIDTHS if w >= m), None)


def _up9(v):
    """ceil((v + 2^-12) * 512) elementwise, float64."""
    return np.ceil((np.asarray(v, np.float64) + 2.0 ** -12) * 512.0)


def quantize_vit(msc, t8, m, width):
    """(match scores (25, width), transitions (8, width) in the kernel's row
    order mm im dm bm mi ii md dd, the profile's cap, emax); column c is node k = c+1."""
    msc = np.asarray(msc, np.float32)
    t8 = np.asarray(t8, np.float32)
    e = np.full((25, width), V_EFLOOR, np.int64)
    real = msc[:, 1:m + 1]
    fin = real > np.float32(-1e30)
    q = np.full(real.shape, V_EFLOOR, np.int64)
    q[fin] = np.maximum(_up9(real[fin]), V_EFLOOR).astype(np.int64)
    e[:, :m] = q
    emax = max(V_EFLOOR, int(q[fin].max())) if fin.any() else V_EFLOOR

    def tq(vals, floor):
        v = np.asarray(vals, np.float32)
        out = np.full(v.shape, floor, np.int64)
        f = v > np.float32(-1e30)
        out[f] = np.maximum(np.minimum(_up9(v[f]), 0.0), floor).astype(np.int64)
        return out

    tr = np.full((8, width), V_TFLOOR, np.int64)
    tr[3, :] = V_BMFLOOR
    k = np.arange(1, m + 1)
    tr[0, :m] = tq(t8[_TMM][k - 1], V_TFLOOR)
    tr[1, :m] = tq(t8[_TIM][k - 1], V_TFLOOR)
    tr[2, :m] = tq(t8[_TDM][k - 1], V_TFLOOR)
    tr[3, :m] = tq(t8[_TBM][k], V_BMFLOOR)
    if m > 1:
        tr[4, :m - 1] = tq(t8[_TMI][1:m], V_TFLOOR)
        tr[5, :m - 1] = tq(t8[_TII][1:m], V_TFLOOR)
    tr[6, :m] = tq(t8[_TMD][k - 1], V_TFLOOR)
    tr[7, :m] = tq(t8[_TDD][k - 1], V_TFLOOR)
    return e, tr, 32767 - emax, emax


def _xsc(L):
    """The multihit length constants (loop, move) the engine computes for a
    target of length L (f32 arithmetic, glibc log in double, as hmmfile.cpp)."""
    f = np.float32
    pmove = f(f(3.0) / f(f(f(L) + f(2.0)) + f(1.0)))
    ploop = f(f(1.0) - pmove)
    return f(_libm.log(float(ploop))), f(_libm.log(float(pmove)))


def vit_bound(msc, t8, m, dsq):
    """The Viterbi pre-screen's bound (f32 nats) for one pair: inf when a row
    maximum exceeded the cap, NaN for an empty target or a profile the
    pre-screen does not take (too wide, or match scores above +16 nats)."""
    L = len(dsq)
    width = vit16_width(m)
    if L == 0 or width is None:
        return np.float32(np.nan)
    e, tr, cap, emax = quantize_vit(msc, t8, m, width)
    if emax >= 8192:
        return np.float32(np.nan)
    tmm, tim, tdm, tbm, tmi, tii, tmd, tdd = tr
    loop, move = _xsc(L)
    tl, tm = _q32_up(loop), _q32_up(move)
    nln2 = int(math.ceil(float(-LN2_F32) * Q32)) + RHO32
    M = np.full(width, V_INIT, np.int64)
    I = np.full(width, V_INIT, np.int64)
    D = np.full(width, V_INIT, np.int64)
    pre = np.full(width, V_INIT, np.int64)
    xn, xj, fin = 0, NEG32, NEG32
    B = max((tm + 2047) >> 11, V_BFLOOR)
    S = np.cumsum(tdd)
    for row, x in enumerate(dsq, 1):
        dleft = np.concatenate(([V_INIT], D[:-1]))
        Mn = np.maximum(np.maximum(pre, dleft + tdm), B + tbm) + e[int(x)]
        mleft = np.concatenate(([V_INIT], Mn[:-1]))
        # D[c] = max(Mn[c-1] + tmd[c], D[c-1] + tdd[c]), D[-1] = Init: a
        # max-plus prefix scan over the column sums of tdd
        a = mleft + tmd
        D = S + np.maximum(np.maximum.accumulate(a - S), V_INIT)
        ileft = np.concatenate(([V_INIT], I[:-1]))
        pre = np.maximum(mleft + tmm, ileft + tim)
        I = np.maximum(Mn + tmi, I + tii)
        M = Mn
        xe = int(M.max())
        if xe > cap:
            return np.float32(np.inf)
        xj = max(xj + tl, xe * 2048 + nln2)
        xn += tl
        xb = max(xn, xj) + tm
        B = max((xb + 2047) >> 11, V_BFLOOR)
        if row == L:
            fin = xj + tm
    return np.float32(_f32_round_up(fin) * np.float32(2.0 ** -20))
