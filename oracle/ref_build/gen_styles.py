"""Write the reference's style_*.h registry headers for the oracle build.

The reference generates these with its csh build step (src/Make.csh:52-219):
for each style family it lists, in `ls` order, the headers that contain the
family's *_CLASS marker and writes `#include "<file>"` lines.  This script does
the same over any number of source directories (the reference's src/ first,
then the oracle's own extra styles), so the reference's build system is never
run.  Test infrastructure only.

usage: python gen_styles.py OUTDIR SRCDIR [SRCDIR ...]
"""
import glob
import os
import sys

FAMILIES = [
    ("style_app.h", "app_*.h", "APP_CLASS"),
    ("style_fft.h", "fft_*.h", "FFT_CLASS"),
    ("style_command.h", "*.h", "COMMAND_CLASS"),
    ("style_diag.h", "diag_*.h", "DIAG_CLASS"),
    ("style_dump.h", "dump_*.h", "DUMP_CLASS"),
    ("style_pair.h", "pair_*.h", "PAIR_CLASS"),
    ("style_region.h", "region_*.h", "REGION_CLASS"),
    ("style_solve.h", "solve_*.h", "SOLVE_CLASS"),
]

# oracle-side styles whose file names do not follow the family glob
EXTRA = {"style_fft.h": ["oracle_slab.h"]}


def main(argv):
    out, srcs = argv[1], argv[2:]
    os.makedirs(out, exist_ok=True)
    for header, pattern, marker in FAMILIES:
        lines = []
        for src in srcs:
            names = sorted(os.path.basename(p) for p in glob.glob(os.path.join(src, pattern)))
            names += [n for n in EXTRA.get(header, []) if os.path.exists(os.path.join(src, n))]
            for name in names:
                if name.startswith("style_"):
                    continue
                with open(os.path.join(src, name), errors="replace") as f:
                    if marker in f.read():
                        lines.append('#include "%s"\n' % name)
        text = "".join(lines)
        path = os.path.join(out, header)
        old = open(path).read() if os.path.exists(path) else None
        if old != text:
            with open(path, "w") as f:
                f.write(text)


if __name__ == "__main__":
    main(sys.argv)
