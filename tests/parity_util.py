"""Helpers shared by the parity tests: near-tie windows and the fit tolerance.

Two FP32 correlations of different FFT algorithms (the engine's and cuFFT's in the
reference) agree to a small absolute error relative to the window's largest value.  Where
two candidates, or a candidate and its neighbour, lie closer than that, their order is
not determined by the inputs: those windows are excluded from exact index and count
comparisons, and reported.
"""
import numpy as np


def near_ties(planes, bx, by, nps, rel=1e-5):
    """(tie_topN, tie_count) masks per window from shifted planes [n][wsy][wsx].

    tie_topN: the window's top Npeak_save list is not determined by the plane at this
    precision -- two of its top Npeak_save+1 local maxima lie within rel (of the window's
    largest maximum) of each other, or a point that would rank among the top Npeak_save is
    within rel of a 4-neighbour, so it may or may not be a local maximum.
    tie_count: some 4-neighbour comparison in the search region is that close (the count
    of maxima is not determined)."""
    n, wsy, wsx = planes.shape
    c = planes[:, by:wsy - by, bx:wsx - bx]
    nbs = (planes[:, by:wsy - by, bx - 1:wsx - bx - 1], planes[:, by:wsy - by, bx + 1:wsx - bx + 1],
           planes[:, by - 1:wsy - by - 1, bx:wsx - bx], planes[:, by + 1:wsy - by + 1, bx:wsx - bx])
    peak = planes.reshape(n, -1).max(1)[:, None, None]
    tol = rel * np.maximum(peak, 1e-30)
    cand = (c > 0)
    close = np.zeros(c.shape, bool)
    for nb in nbs:
        cand &= c >= nb
        close |= np.abs(c - nb) <= tol
    tie_count = close.reshape(n, -1).any(1)
    vals = np.where(cand, c, -np.inf).reshape(n, -1)
    top = -np.sort(-vals, axis=1)[:, :nps + 1]
    both = np.isfinite(top[:, 1:]) & np.isfinite(top[:, :-1])
    with np.errstate(invalid="ignore"):  # -inf - -inf where a window has few maxima
        tie_top = (both & (np.abs(np.diff(top, axis=1)) <= rel * top[:, :1])).any(1)
    # the Npeak_save-th maximum (or 0 when there are fewer): a near-tie point above it ranks
    kth = top[:, min(nps, top.shape[1]) - 1]
    floor = np.where(np.isfinite(kth), kth - tol[:, 0, 0], 0.0)[:, None, None]
    tie_rank = (close & (c > 0) & (c >= floor)).reshape(n, -1).any(1)
    tie_top |= tie_rank
    return tie_top, tie_count | tie_top


def fit_tolerance(planes, idx, wsx, rel_cc=1e-5, base=1e-3, safety=1.0):
    """Per-candidate bound on |engine - reference| of the 3-point Gaussian fit, per axis.
    delta = num / (2 den), num = ln f- - ln f+, den = ln f- + ln f+ - 2 ln f0; two FP32 FFTs
    of different algorithms agree to about rel_cc of the window's largest value (absolute),
    so a value c carries a log error rel_cc * max / c; the reference also rounds its FP32
    logs (1 ulp each) and sums.  Propagated: |d delta| <= (|delta| e_den + e_num / 2) /
    (|den| - e_den), times `safety`, plus `base`; inf where the denominator's sign is not
    determined.  With rel_cc = 0 it bounds two fits of the same plane (FP32 against FP64
    logs)."""
    n = planes.shape[0]
    flat = planes.reshape(n, -1)
    size = flat.shape[1]
    cmax = flat.max(1)[:, None]
    out = []
    for axis in (1, wsx):
        t = np.full(idx.shape, base)
        ok = (idx >= axis) & (idx + axis < size)
        li = np.where(ok, idx, axis)
        c0 = np.take_along_axis(flat, li - axis, 1).astype(np.float64)
        c1 = np.take_along_axis(flat, li, 1).astype(np.float64)
        c2 = np.take_along_axis(flat, li + axis, 1).astype(np.float64)
        pos = ok & (c0 > 0) & (c1 > 0) & (c2 > 0)
        t[ok & ~pos] = np.inf
        with np.errstate(divide="ignore", invalid="ignore"):
            f0, f1, f2 = np.log(c0), np.log(c1), np.log(c2)
            den = f0 + f2 - 2 * f1
            e0, e1, e2 = rel_cc * cmax / c0, rel_cc * cmax / c1, rel_cc * cmax / c2
            e_num = e0 + e2 + 2.0 ** -23 * (np.abs(f0) + np.abs(f2))
            e_den = e0 + e2 + 2 * e1 + 2.0 ** -22 * (np.abs(f0) + np.abs(f2) + 2 * np.abs(f1))
            delta = (f0 - f2) / den / 2
            tt = base + safety * (np.abs(delta) * e_den + e_num / 2) / (np.abs(den) - e_den)
        undetermined = pos & (np.abs(den) <= e_den)
        t[pos & ~undetermined] = tt[pos & ~undetermined]
        t[undetermined] = np.inf
        out.append(t)
    return out


def fit_undetermined(planes, idx, wsx, rel=1e-5):
    """Candidates whose 3-point fit reads a value within rel (of the window's largest
    value) of zero: the log of a value at the planes' error level may be finite on one side
    and -inf on the other, so the fit's validity is not determined by the inputs."""
    n = planes.shape[0]
    flat = planes.reshape(n, -1)
    size = flat.shape[1]
    tol = rel * flat.max(1)[:, None]
    out = np.zeros(idx.shape, bool)
    for o in (0, -1, 1, -wsx, wsx):
        j = idx + o
        inside = (idx >= 0) & (j >= 0) & (j < size)
        val = np.take_along_axis(flat, np.where(inside, j, 0), 1)
        out |= inside & (val <= tol)
    return out

