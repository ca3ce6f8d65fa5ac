"""Makes tests/golden/shortpulse_table.npz from the reference's own short-pulse
test program (test/testshortpulse.cpp, built by `make -C oracle shortpulse`
into oracle/_ref/testshortpulse): it evaluates ShortPulseInjectSourceFunc's
Efunc and Bfunc (bx, by) with setParam(length 1e6, width 2, om0 2, Shift 0,
Phase 0, amp 1, eps 1) on x = -5..5 (step 0.05), y = z = 0, t = 0..8 (step
0.025) and prints Re and Im of each into debug1.out .. debug6.out.  Every
fourth x and every fourth t are kept (51 x 81 points).

    python tests/golden/make_shortpulse_table.py
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "..", "..", "oracle", "_ref", "testshortpulse")


def read_table(path):
    rows = [ln.split() for ln in open(path) if ln.strip()]
    return np.array(rows, dtype=np.float64)  # x, t, value


def main():
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([os.path.abspath(BIN)], cwd=d, check=True, stderr=subprocess.DEVNULL)
        cols = [read_table(os.path.join(d, f"debug{q}.out")) for q in range(1, 7)]
    xt = cols[0][:, :2]
    for c in cols[1:]:
        assert np.array_equal(c[:, :2], xt)
    nt = int(np.sum(xt[:, 0] == xt[0, 0]))
    nx = len(xt) // nt
    vals = np.stack([c[:, 2] for c in cols], axis=1).reshape(nx, nt, 6)
    keep = vals[::4, ::4]
    x = xt[::nt, 0][::4]
    t = xt[:nt, 1][::4]
    np.savez_compressed(os.path.join(HERE, "shortpulse_table.npz"), x=x, t=t, values=keep,
                        params=np.array([1e6, 2.0, 2.0, 0.0, 1.0]))
    print("x", len(x), "t", len(t))


if __name__ == "__main__":
    main()
