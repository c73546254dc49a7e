"""Generates zm_fft2_<dtype>_<dir>.cu: the size-specialised fused passes and their
dispatch tables.  Each (log2 VEC, log2 M) pair lists variants (cluster size CL, lines
per tile TL, threads NT[, "p" = persistent forward pass with bulk-copy prefetch]); the
plan's `variant` picks one; "k3" marks the three-stage 512-thread pass of zm_fft3.cuh
for complex64 lines of 2^14 points ("k3p": its persistent form with asynchronous copies
of the next line; "k3c": the forward y pass on buddy-line CTA pairs); "t" marks the
persistent form of the fused pass whose next tile's first-phase points are staged in
tensor memory (one CTA per SM).  Variant 0, the default, is
the fastest one measured on B200 at the sizes the table was tuned on; zm_plan_autotune
re-measures them for a plan."""
VARIANTS = {
    "c64": {
        (4, 4): [(1, 32, 512)], (4, 5): [(1, 16, 512)], (4, 6): [(1, 8, 512), (1, 4, 256)],
        (2, 7): [(1, 8, 256), (1, 16, 512), (1, 32, 1024), (1, 4, 128)], (5, 6): [(1, 4, 512)],
        (5, 7): [(1, 2, 512), (2, 2, 256), (2, 4, 512), (1, 1, 256), (1, 4, 1024)],
        (4, 8): [(1, 2, 512), (2, 4, 512), (1, 1, 256), (1, 4, 1024)],
        (5, 8): [(2, 2, 512), (1, 1, 512), (2, 1, 256), (4, 4, 512), (2, 4, 1024), (1, 2, 1024)],
        (6, 7): [(2, 2, 512), (1, 1, 512), (1, 2, 1024)],
        (6, 8): [(4, 2, 512), (2, 1, 512), (1, 1, 1024), (8, 4, 512), (4, 4, 1024), (4, 2, 512, "p"),
                 (1, 1, 512, "k3"), (1, 1, 512, "k3p"), (1, 1, 512, "k3c")],
    },
    "c128": {
        (4, 4): [(1, 16, 256)], (4, 5): [(1, 8, 256)], (4, 6): [(1, 4, 256)], (2, 7): [(1, 8, 256), (1, 4, 128), (1, 16, 512)],
        (5, 6): [(1, 2, 256)], (5, 7): [(1, 1, 256), (2, 2, 256)], (4, 8): [(1, 1, 256), (2, 2, 256)],
        (5, 8): [(1, 1, 512), (2, 1, 256)], (6, 7): [(2, 1, 256), (1, 1, 512)],
        (6, 8): [(2, 1, 512), (4, 1, 256), (4, 2, 512), (2, 1, 512, "t"), (4, 2, 512, "t")],
    },
}
# Out-of-place 2D forward configurations (used when the caller passes a workspace and the
# plan runs its default variant): x pass variant, y pass variant, log2 of the row
# interleave of the intermediate.  Measured on B200 at N = 16384, P = 4, B = 64 (c64):
# x pass on the persistent three-stage kernel (1.21 ms), y pass on buddy-line CTA pairs
# of the three-stage kernel reading the 8-row interleave (1.77 ms; one line per CTA
# 1.81): 2.97 ms per forward transform against 4.61 for the in-place default.
# complex128 (6, 8): a 16-row interleave (G = VP), so that the x pass on one-line tiles
# writes runs of 16 elements (256 bytes) -- with the plain layout it wrote each 16-byte
# element into a 32-byte sector of its own (5.16 ms) -- and the y pass reads its line 16
# elements apart on the persistent tensor-memory-staged tiles (variant 3), which hide the
# wait for those scattered reads: x 3.30 + y 3.70 = 6.97 ms per forward transform, against
# 7.86 (two-line x tiles on clusters of four writing the 2-row interleave) and 8.51.
FWD_OOP = {
    "c64": {(6, 8): (7, 8, 3), (5, 8): (5, 5, 1), (6, 7): (2, 2, 1)},
    "c128": {(6, 8): (0, 3, 4)},
}
# Out-of-place 2D inverse configurations (caller workspace, default variant): y pass
# variant (frequency side -> work), x pass variant (work -> vector side), log2 of the
# interleave, and "q" for groups of y positions interleaved instead of x-frequency rows
# (three-stage kernels only).  Measured on B200 at N = 16384, P = 4, B = 64 (c64): both
# passes on the persistent three-stage kernel, the y pass writing runs of 4 y positions
# (whole 32-byte sectors), the x pass reading its line 4 elements apart (four lanes per
# 128-byte line): 1.67 + 1.46 = 3.12 ms per inverse transform, against 3.24 for the
# row-interleaved intermediate (8-element runs: 1.62 + 1.79; 16-byte runs: partial
# sectors, 2.2 ms and up for the y pass).
# complex128 (6, 8): both passes on the persistent tensor-memory-staged tiles (variant 3),
# plain REPACK intermediate: 6.11 ms against 6.81 (the x pass, whose strided frequency-side
# reads wait longest, 4.04 -> 3.39 ms; the y pass unchanged).
INV_OOP = {
    "c64": {(6, 8): (7, 7, 2, "q")},
    "c128": {(6, 8): (3, 3, 0)},
}
T = {"c64": "float", "c128": "double"}
for dt, table in VARIANTS.items():
    for inv in (False, True):
        d = "inv" if inv else "fwd"
        L = [f"// zm_fft2_{dt}_{d}.cu -- generated by gen_fused.py: size-specialised fused axis passes,",
             f"// {dt}, {'inverse' if inv else 'forward'} direction (kernel template in zm_fft2.cuh).",
             '#include "zm_internal.h"', '#include "zm_lines.cuh"', '#include "zm_fft2.cuh"',
             '#include "zm_fft3.cuh"', "",
             "namespace zm {", "",
             f"cudaError_t launch_fused_{dt}_{d}(const LineParams &prm, cudaStream_t st, bool *handled) {{",
             "    *handled = true;",
             "    switch ((prm.g.logVEC << 16) | (prm.g.logM << 8) | prm.variant) {"]
        for (lv, lm), vs in table.items():
            for vi, v in enumerate(vs):
                cl, tl, nt = v[:3]
                pers = "true" if len(v) > 3 and v[3] == "p" else "false"
                tms = ", true" if len(v) > 3 and v[3] == "t" else ""
                if len(v) > 3 and v[3] in ("k3", "k3p", "k3c"):
                    L.append(f"    case ({lv} << 16) | ({lm} << 8) | {vi}: "
                             f"return launch_k3<{lv}, {lm}, {'true' if inv else 'false'}, "
                             f"{'true' if v[3] == 'k3p' else 'false'}, "
                             f"{'true' if v[3] == 'k3c' else 'false'}>(prm, st);")
                    continue
                L.append(f"    case ({lv} << 16) | ({lm} << 8) | {vi}: "
                         f"return launch_fused<{T[dt]}, {lv}, {lm}, {cl}, {tl}, {nt}, {'true' if inv else 'false'}, {pers}{tms}>(prm, st);")
        L += ["    default: break;", "    }", "    *handled = false;", "    return cudaSuccess;", "}", ""]
        if not inv:
            L += [f"int fused_variants_{dt}(int logvec, int logm) {{", "    switch ((logvec << 8) | logm) {"]
            for (lv, lm), vs in table.items():
                L.append(f"    case ({lv} << 8) | {lm}: return {len(vs)};")
            L += ["    default: return 0;", "    }", "}", ""]
            # log2 of the widest row interleave G of the 2D intermediate a variant can run
            # on: G <= 4 lines per tile and G | TL (a group of G rows is read and written
            # by one tile, so the in-place y pass is race-free), two row stages (the
            # vector side moves through registers, not 16-byte copies) and at least G
            # columns per CTA; 0 = plain REPACK layout
            L += [f"int fused_interleave_lg_{dt}(int logvec, int logm, int variant) {{",
                  "    switch ((logvec << 16) | (logm << 8) | variant) {"]
            for (lv, lm), vs in table.items():
                for vi, v in enumerate(vs):
                    cl, tl, nt = v[:3]
                    vec, n = 1 << lv, 1 << (lv + lm)
                    ept = tl * n // (cl * nt)
                    ra2 = vec // min(vec, ept)
                    g = min(tl, 4)
                    while g > 1 and vec // cl < g:
                        g //= 2
                    if g >= 2 and ra2 > 1:
                        L.append(f"    case ({lv} << 16) | ({lm} << 8) | {vi}: return {g.bit_length() - 1};")
            L += ["    default: return 0;", "    }", "}", ""]
            for name, oop in (("fwd", FWD_OOP), ("inv", INV_OOP)):
                L += [f"int fused_{name}_oop_{dt}(int logvec, int logm, int *vx, int *vy, int *lg, int *qint) {{",
                      "    switch ((logvec << 8) | logm) {"]
                for (lv, lm), cfg in oop[dt].items():
                    v1, v2, lg = cfg[:3]
                    q = 1 if len(cfg) > 3 and cfg[3] == "q" else 0
                    a, b = (v1, v2) if name == "fwd" else (v2, v1)
                    L.append(f"    case ({lv} << 8) | {lm}: *vx = {a}; *vy = {b}; *lg = {lg}; *qint = {q}; return 1;")
                L += ["    default: return 0;", "    }", "}", ""]
        L += ["}  // namespace zm", ""]
        open(f"zm_fft2_{dt}_{d}.cu", "w").write("\n".join(L))
