"""Writes kernels_mixcols_t0.cu .. kernels_mixcols_t7.cu: the compiled
mixed-radix column tiles (gfft_mixcols.cuh) of every 7-smooth column length
48 <= L <= 1024, spread over eight files so nvcc builds them in parallel; and
kernels_mixrows_t0.cu .. kernels_mixrows_t7.cu: the same schedules in rows
mode (k_mix_rows: whole contiguous transforms of every table length, several
per CTA, the single-pass plans of those lengths), plus three-stage schedules
for the 7-smooth lengths 1025..12288 that are not powers of two (complex128
up to 6144, the shared memory one transform can have); and
kernels_mixbs_t0.cu .. kernels_mixbs_t2.cu: the Bluestein chain's passes
(gfft_mixbs.cuh) for the column lengths its FFT lengths M = M1 x M2 are built
from (the 7-smooth multiples of 16 up to 512, whose products come within
1.5% of the best 7-smooth M on average, less 48, 64 and 96, which never make
the smallest M >= 2n - 1 for an n beyond the one-CTA Bluestein range), with
the same schedules.

Schedule rule, from timing the candidates on a B200 (two stages against three
and four, several tile widths and occupancies, at L = 100..1000):
  * two stages L = a * b, the larger radix a first and as small as it can be
    (both radices 7-smooth, at most 49, or a power of two up to 64): fewer
    stages mean fewer shared-memory exchanges and barriers;
  * b threads per column (a thread owns one butterfly of radix a and
    ceil(a / b) of radix b), or a threads ("wide": one butterfly of radix b;
    b of the a threads take one of radix a, so no thread holds more than a
    values) for the lengths in WIDE, where timing every table entry both ways
    (pass 1 and 2 over L x L complex elements, 256 MiB batches) showed the
    wide form at least 3% faster: mostly radices within a factor of 1.5 of
    each other; the narrow form stays ahead where a is much larger than b or,
    in complex128, a >= 35;
  * tiles of 16 columns (complex64) / 8 (complex128) below L = 500, else 8 / 4;
  * resident CTAs per SM asked of the register allocation (MINB): as many as
    keep an estimate of the registers a thread needs (its largest stage's
    values at two registers each, or four with a 1.3 margin for complex128,
    plus 40), fit 1024 threads and 200 KB of shared memory per SM, at most 8.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PARTS = 8
BS_PARTS = 3
ROW_PARTS = 8
ROWS3_MAX = {8: 12288, 16: 6144}  # longest three-stage rows length per element size


def smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def radix_ok(r):
    return r >= 2 and smooth7(r) and (r <= 49 or (r & (r - 1) == 0 and r <= 64))


def schedule(L):
    best = None
    for b in range(2, int(L ** 0.5) + 1):
        if L % b == 0 and radix_ok(b) and radix_ok(L // b):
            a = L // b
            if best is None or a < best[0]:
                best = (a, b)
    if best is None:
        raise ValueError(f"no two-stage schedule for {L}")
    return best


# Lengths whose two radices do not divide and that run faster with a threads
# per column, per element size (bytes).
WIDE = {
    8: {56, 72, 90, 108, 120, 168, 180, 192, 210, 224, 240, 270, 288, 360, 378, 420, 480, 500, 504, 525, 567,
        588, 600, 630, 648, 672, 675, 700, 720, 750, 756, 800, 810, 840, 864, 875, 896, 945, 960, 972, 980, 1008},
    16: {48, 54, 56, 63, 72, 80, 90, 108, 120, 126, 135, 140, 150, 160, 168, 180, 210, 224, 240, 252, 270, 280,
         288, 300, 315, 320, 336, 360, 378, 420, 432, 450, 480, 486, 500, 504, 525, 540, 560, 567, 588, 600, 630,
         640, 648, 672, 675, 700, 720, 750, 756, 768, 800, 810, 840, 864, 896, 960},
}


def threads(L, sched, wide):
    """Threads per column: L / max radix, or L / min radix (wide)."""
    return L // (min(sched) if wide else max(sched))


def vmax(L, sched, T):
    return max(-(-(L // r) // T) * r for r in sched)


def minb(L, sched, nc, es, T, extra=0):
    tpb = T * nc
    tpbw = -(-tpb // 32) * 32
    per = 2 * (es // 8)  # registers per complex value
    regs = int(per * vmax(L, sched, T) * (1.0 if es == 8 else 1.3)) + 40 + extra
    pitch = nc + 1 if nc >= 16 else nc
    smem = max(L * pitch, nc * (L | 1)) * es
    k = 1
    while (k < 8 and 65536 // ((k + 1) * tpbw) >= regs and (k + 1) * tpb <= 1024
           and (k + 1) * smem <= 200 * 1024):
        k += 1
    return k


# Lengths whose three-stage schedule (schedule3, 8 columns per tile) beat
# the two-stage one when both forms of the long column lengths were timed,
# per element size: complex64 480 (24 x 20 on a thread per radix-20
# butterfly, one CTA per SM) 1.11x in pass 1 and 1.22x in pass 2; for every
# other length from 240 to 1024 the two-stage form was 4-27% faster.
# Value: resident CTAs per SM asked of pass 1 and of pass 2.
THREE = {8: {480: (3, 4)}, 16: {}}
# Complex128 lengths whose pass 2 alone ran faster on the three-stage
# schedule (pass 1 kept the two-stage one at every length): 336 1.16x, 512
# 1.13x, 1000 1.10x, 768 1.08x.  Value: (tile width, resident CTAs per SM).
THREE2 = {8: {}, 16: {336: (8, 3), 512: (8, 2), 768: (4, 3), 1000: (4, 2)}}


def plan(L, es, extra=0, pass_=1):
    """(radices, tile width, MINB, threads per column or 0) of one column
    pass (1 or 2); `extra` registers per thread added to the occupancy
    estimate."""
    if L in THREE[es]:
        return schedule3(L), 8, THREE[es][L][pass_ - 1], 0
    if pass_ == 2 and L in THREE2[es]:
        nc, mb = THREE2[es][L]
        return schedule3(L), nc, mb, 0
    return plan2(L, es, extra)


def plan2(L, es, extra=0):
    """The two-stage plan of plan()."""
    sched = schedule(L)
    nc = (16 if L < 500 else 8) if es == 8 else (8 if L < 500 else 4)
    wide = sched[0] % sched[1] != 0 and L in WIDE[es]
    T = threads(L, sched, wide)
    return sched, nc, minb(L, sched, nc, es, T, extra), T if wide else 0


def schedule3(L):
    """Three stages L = a * b * c, a >= b >= c, the largest radix as small as
    it can be, then the smallest as large."""
    best = None
    for a in range(2, 65):
        if L % a or not radix_ok(a):
            continue
        for b in range(2, a + 1):
            if (L // a) % b or not radix_ok(b):
                continue
            c = L // a // b
            if 2 <= c <= b and radix_ok(c) and (best is None or (a, -c) < best[0]):
                best = ((a, -c), (a, b, c))
    if best is None:
        raise ValueError(f"no three-stage schedule for {L}")
    return best[1]


def rows3_lengths(es):
    return [L for L in range(1025, ROWS3_MAX[es] + 1) if smooth7(L) and L & (L - 1)]


def rows_pitch(L, sched):
    """Shared-memory elements per transform in rows mode (MixTileRows::LP)."""
    r0 = sched[0]
    return (L + (L - 1) // r0 + 1 if r0 % 2 == 0 else L) | 1


def rows_plan(L, es):
    """Rows mode: the column schedule and thread layout; transforms per CTA
    (a power of two) as many as keep the CTA within 512 threads and 64 KB of
    shared memory; resident CTAs per SM by the same register estimate, up to
    2048 threads and 200 KB per SM."""
    if L <= 1024:
        sched, _, _, tt = plan2(L, es)
    else:
        sched, tt = schedule3(L), 0
    T = tt if tt else L // max(sched)
    assert T <= 1024, (L, sched)
    lp = rows_pitch(L, sched)
    nc = 1
    while nc < 64 and T * nc * 2 <= 512 and 2 * nc * lp * es <= 64 * 1024:
        nc *= 2
    tpb = T * nc
    tpbw = -(-tpb // 32) * 32
    regs = int(2 * (es // 8) * vmax(L, sched, T) * (1.0 if es == 8 else 1.3)) + 40
    smem = nc * lp * es
    k = 1
    while (k < 8 and 65536 // ((k + 1) * tpbw) >= regs and (k + 1) * tpb <= 2048
           and (k + 1) * smem <= 200 * 1024):
        k += 1
    return sched, nc, k, tt


def rows_cfg(L, es):
    sched, nc, mb, tt = rows_plan(L, es)
    s = ", ".join(str(r) for r in sched)
    return f"MixCfg<MixSched<{s}>, {nc}, {mb}, {tt}>"


def cfg(L, es, extra=0, pass_=1):
    sched, nc, mb, tt = plan(L, es, extra, pass_)
    s = ", ".join(str(r) for r in sched)
    return f"MixCfg<MixSched<{s}>, {nc}, {mb}, {tt}>"


def bs_lengths():
    return [L for L in range(48, 513) if smooth7(L) and L % 16 == 0 and L not in (48, 64, 96)]


def main(out=HERE):
    lengths = [L for L in range(48, 1025) if smooth7(L)]
    parts = [[] for _ in range(PARTS)]
    for i, L in enumerate(lengths):
        f1, f2 = cfg(L, 8), cfg(L, 8, pass_=2)
        d1, d2 = cfg(L, 16), cfg(L, 16, pass_=2)
        parts[i % PARTS].append(f"  v.push_back(mix_entry<{f1},\n                         {f2},\n"
                                f"                         {d1},\n                         {d2}>());  // {L}\n")
    for k, body in enumerate(parts):
        with open(os.path.join(out, f"kernels_mixcols_t{k}.cu"), "w") as fh:
            fh.write("// Generated by gen_mixcols.py; do not edit.\n"
                     "#include \"kernels_mixcols.cuh\"\n\nnamespace gfft {\n\n"
                     f"void mix_part_{k}(std::vector<MixEntry>& v) {{\n" + "".join(body) + "}\n\n}  // namespace gfft\n")
    rparts = [[] for _ in range(ROW_PARTS)]
    for i, L in enumerate(lengths + rows3_lengths(8)):
        if L <= 1024 or L in rows3_lengths(16):
            e = f"  v.push_back(mix_rows_entry<{rows_cfg(L, 8)},\n                              {rows_cfg(L, 16)}>());  // {L}\n"
        else:
            e = f"  v.push_back(mix_rows_entry64<{rows_cfg(L, 8)}>());  // {L}\n"
        rparts[i % ROW_PARTS].append(e)
    for k, body in enumerate(rparts):
        with open(os.path.join(out, f"kernels_mixrows_t{k}.cu"), "w") as fh:
            fh.write("// Generated by gen_mixcols.py; do not edit.\n"
                     "#include \"kernels_mixcols.cuh\"\n\nnamespace gfft {\n\n"
                     f"void mix_rows_part_{k}(std::vector<MixRowsEntry>& v) {{\n" + "".join(body) + "}\n\n}  // namespace gfft\n")
    bparts = [[] for _ in range(BS_PARTS)]
    for i, L in enumerate(bs_lengths()):
        bparts[i % BS_PARTS].append(f"  v.push_back(mix_bs_entry<{cfg(L, 8)},\n                            {cfg(L, 16)}>());  // {L}\n")
    for k, body in enumerate(bparts):
        with open(os.path.join(out, f"kernels_mixbs_t{k}.cu"), "w") as fh:
            fh.write("// Generated by gen_mixcols.py; do not edit.\n"
                     "#include \"kernels_mixcols.cuh\"\n\nnamespace gfft {\n\n"
                     f"void mix_bs_part_{k}(std::vector<MixBsEntry>& v) {{\n" + "".join(body) + "}\n\n}  // namespace gfft\n")
    print(len(lengths), "lengths,", len(rows3_lengths(8)), "three-stage rows lengths,", len(bs_lengths()), "Bluestein lengths")


if __name__ == "__main__":
    main()
