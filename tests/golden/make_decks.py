"""Write the deck fixtures of tests/test_gpu_reference_app.py from the
reference's own example decks (src/in.fcc-pfdd, src/in.bcc-pfdd).

Each deck is kept line for line (commented-out lines dropped) with three
changes: max_iter 5000 -> MAX_ITER (a test-sized run; tol kept), the dump
written every DUMP_EVERY steps to dump.txt, and, for the `b200` variant, the
two style lines swapped to the library's drop-in styles:
    fft_style fftw_slab ...  ->  fft_style b200 ... precision fp64
    solve_style GL ...       ->  solve_style GLgpu ...
Run here (the reference tree is not on the GPU machines):
    python tests/golden/make_decks.py /root/reference/src
"""
import os
import sys

MAX_ITER = 40
DUMP_EVERY = 10
HERE = os.path.dirname(os.path.abspath(__file__))


def derive(text, variant):
    out = []
    for line in text.splitlines():
        s = line.strip()
        if not s or s.startswith("#"):
            continue
        w = s.split()
        if w[0] == "solve_style":
            w = [("GLgpu" if variant == "b200" else w[1]) if i == 1 else
                 (str(MAX_ITER) if i > 0 and w[i - 1] == "max_iter" else x) for i, x in enumerate(w)]
            w.insert(0, "solve_style")
            w.pop(1)
        elif w[0] == "fft_style" and variant == "b200":
            s = s.split("#")[0].strip()
            w = s.split()
            w[1] = "b200"
            w += ["precision", "fp64"]
        elif w[0] == "dump":
            w[3] = str(DUMP_EVERY)
            w[4] = "dump.txt"
        else:
            w = s.split("#")[0].split()
        out.append(" ".join(w))
    return "\n".join(out) + "\n"


def main(src):
    os.makedirs(os.path.join(HERE, "decks"), exist_ok=True)
    for name in ("in.fcc-pfdd", "in.bcc-pfdd"):
        text = open(os.path.join(src, name)).read()
        for variant in ("ref", "b200"):
            path = os.path.join(HERE, "decks", "%s.%s" % (name, variant))
            with open(path, "w") as f:
                f.write(derive(text, variant))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")
