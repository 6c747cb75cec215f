"""Generates fft_layouts.h: the padded shared-memory layouts of the Stockham
exchanges of fft_core.cuh (SmPencil), chosen by counting bank wavefronts.

Exchange S of a plan (written by stage S: radix R, span Ns; read by stage S+1:
radix R2) stores row r either at r + (r // X) * pad, X = Ns * R (pad >= 0), or
at the XOR swizzle r ^ ((r >> 2) & (G - 1)) (recorded as pad -1; G rows of one
128-byte bank line).  For every compiled length, values-per-thread E, element
size and direction, the layout with the fewest shared-memory wavefronts over the
exchange's writes and reads is recorded (ties go to the padded layout, whose
addresses need no per-access arithmetic); where several pencils share a warp, so
is the pencil pitch with the fewest wavefronts.  Wavefronts are counted per
phase of a warp access: 16 lanes for 8-byte and 8 lanes for 16-byte elements,
each phase taking as many wavefronts as its busiest 4-byte bank.  Run: python gen_layouts.py (writes the
header beside this file)."""
import math
import os
import sys

LENGTHS = (48, 72, 96, 144, 192, 288, 384, 768, 1536)
EVALUES = (4, 6, 8, 12, 16, 24, 32, 48)
RADICES = (12, 8, 6, 4, 3, 2)      # greedy order of fft_core.cuh pick_radix
PAD_MAX = 6


def plan(L, E, inv):
    rs, rem = [], L
    while rem > 1:
        r = next((r for r in RADICES if rem % r == 0 and E % r == 0), 0)
        if r == 0:
            return None
        rs.append(r)
        rem //= r
    return rs[::-1] if inv else rs


def wavefronts(addrs, wpl):
    lanes = 16 if wpl == 2 else 8
    tot = 0
    for ph in range(0, 32, lanes):
        c = [0] * 32
        for a in addrs[ph:ph + lanes]:
            for w in range(wpl):
                c[(a + w) % 32] += 1
        tot += max(c)
    return tot


def place(row, X, pad, wpl):
    if pad >= 0:
        return row + (row // X) * pad
    G = 16 if wpl == 2 else 8
    return row ^ ((row >> 2) & (G - 1))


def cost(L, E, rs, S, pad, pitch, wpl):
    Q = L // E
    R, R2 = rs[S], rs[S + 1]
    Ns = math.prod(rs[:S])
    X = Ns * R
    lay = lambda row: place(row, X, pad, wpl)  # noqa: E731
    c = 0
    for m in range(E // R):
        for r in range(R):
            a = []
            for t in range(32):
                p, q = divmod(t, Q)
                j = q + Q * m
                a.append((p * pitch + lay((j // Ns) * X + j % Ns + r * Ns)) * wpl)
            c += wavefronts(a, wpl)
    for m in range(E // R2):
        for r in range(R2):
            a = []
            for t in range(32):
                p, q = divmod(t, Q)
                a.append((p * pitch + lay(q + Q * m + r * (L // R2))) * wpl)
            c += wavefronts(a, wpl)
    return c


def extent(L, rs, S, pad, wpl=2):
    if pad < 0:
        G = 16 if wpl == 2 else 8
        return (L + G - 1) // G * G
    return L + (L // (math.prod(rs[:S]) * rs[S])) * pad


def best_pad(L, E, rs, S, pitch, wpl, lim):
    best, bc = -1, cost(L, E, rs, S, -1, pitch, wpl)
    for pad in range(0, PAD_MAX + 1):
        if extent(L, rs, S, pad) > lim:
            break
        c = cost(L, E, rs, S, pad, pitch, wpl)
        if c < bc or (c == bc and best < 0):
            best, bc = pad, c
    return best


def layout(L, E, wpl):
    """(pitch, {(inv, S): pad}) of one (length, E, element size)."""
    lim = L + L // 2
    Q = L // E
    plans = {inv: plan(L, E, inv) for inv in (True, False)}
    if Q >= 32:
        pads = {(inv, S): best_pad(L, E, rs, S, 0, wpl, lim) for inv, rs in plans.items() for S in range(len(rs) - 1)}
        pitch = max([L] + [extent(L, plans[inv], S, p, wpl) for (inv, S), p in pads.items()])
        return pitch, pads
    best = None
    for d in range(16):
        pitch = lim + d
        pads = {(inv, S): best_pad(L, E, rs, S, pitch, wpl, lim) for inv, rs in plans.items() for S in range(len(rs) - 1)}
        c = sum(cost(L, E, plans[inv], S, p, pitch, wpl) for (inv, S), p in pads.items())
        if best is None or c < best[0]:
            best = (c, pitch, pads)
    return best[1], best[2]


def generate():
    pads, pitches = [], []
    for wpl in (2, 4):
        for L in LENGTHS:
            for E in EVALUES:
                if L % E or plan(L, E, False) is None:
                    continue
                pitch, pd = layout(L, E, wpl)
                pitches.append((wpl, L, E, pitch))
                for (inv, S), p in sorted(pd.items()):
                    pads.append((wpl, L, E, int(inv), S, p))
    out = ["// Generated by gen_layouts.py -- do not edit.  Padded exchange layouts of",
           "// SmPencil (fft_core.cuh): pad per exchange and pencil pitch, in rows.",
           "#pragma once", "", "namespace spns {", "namespace exch {",
           "struct PadEntry { int wpl, L, E, inv, S, pad; };",
           "struct PitchEntry { int wpl, L, E, pitch; };",
           "constexpr PadEntry kPads[] = {"]
    out += ["    {%d, %d, %d, %d, %d, %d}," % e for e in pads]
    out += ["};", "constexpr PitchEntry kPitches[] = {"]
    out += ["    {%d, %d, %d, %d}," % e for e in pitches]
    out += ["};",
            "constexpr int table_pad(int wpl, int L, int E, bool inv, int S) {",
            "    for (const PadEntry &e : kPads)",
            "        if (e.wpl == wpl && e.L == L && e.E == E && e.inv == (inv ? 1 : 0) && e.S == S) return e.pad;",
            "    return -1;",
            "}",
            "constexpr int table_pitch(int wpl, int L, int E) {",
            "    for (const PitchEntry &e : kPitches)",
            "        if (e.wpl == wpl && e.L == L && e.E == E) return e.pitch;",
            "    return -1;",
            "}",
            "} // namespace exch", "} // namespace spns", ""]
    return "\n".join(out)


if __name__ == "__main__":
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fft_layouts.h")
    text = generate()
    if len(sys.argv) > 1 and sys.argv[1] == "--check":
        sys.exit(0 if open(path).read() == text else 1)
    open(path, "w").write(text)
    print("wrote", path)
