#!/usr/bin/env python3
"""Time the reference's own CUDA build (complex128, cuFFT) on the local GPU.

Runs oracle/_ref/gpe_ref_trace (built by oracle/ref.mk from the reference
sources; test infrastructure) on a real-time input of the headline size.  The
binary reports the device-synchronised wall time of the reference's own
evolution loop (ref_loop_seconds); the difference of two runs with niter = n1
and n2 cancels what the loop does once (the initial and final copies).
Process start-up, cuFFT plans and file output are outside the loop; status
output, frame output and tracing are pushed beyond niter.

Usage (on a GPU host):  python oracle/time_ref_build.py [--n 128] [--n1 500] [--n2 5500] [--imag]
Prints one JSON line: steps/s of the reference build's real-time RK4 loop, or
with --imag of its imaginary-time (heavy-ball) loop.
"""
import argparse
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "gpe_ref_trace")

INPUT = """hamiltonian     "bec"
outprefix       "{out}rt_"
treal           {treal}
read_vext       false
vprefix         "{out}"
read_psi        false
inprefix        "{out}"
t2component     false
npart           1
mass            86.9090
tvseed          true
nseed           2
aseed           0.05
a               100.4
quench_f0       1.1
quench_f1       1.1
quench_f2       1.1
quench_t1       0.0
quench_t2       0.0
quench_t3       0.0
omx             30.0
omy             30.0
omz             60.0
xmax            10.0
ymax            10.0
zmax            10.0
nx              {n}
ny              {n}
nz              {n}
dt              0.002
niter           {niter}
epsilon_e       1E-30
itmod           100000000
itStatMod       100000000
trace_every     100000000
time0           0.0
rand_pct        0.0
crand_pct       0.0
trotate         false
omega           0.0
tpi_vortex      false
api_prc         0.0
beta            0.0
rndseed         367
"""


def run(n, niter, work, imag=False):
    fn = os.path.join(work, f"in_{niter}.txt")
    with open(fn, "w") as f:
        f.write(INPUT.format(out=work + "/", n=n, niter=niter, treal="false" if imag else "true"))
    r = subprocess.run([BIN, fn], capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"reference build failed ({r.returncode}): {r.stderr[-500:]}")
    for line in r.stderr.splitlines():
        if line.startswith("ref_loop_seconds "):
            return float(line.split()[1])
    raise RuntimeError("reference build printed no ref_loop_seconds line")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--n1", type=int, default=500)
    ap.add_argument("--n2", type=int, default=5500)
    ap.add_argument("--repeat", type=int, default=5)
    ap.add_argument("--imag", action="store_true",
                    help="time the imaginary-time (heavy-ball) loop instead of real-time RK4")
    args = ap.parse_args()
    with tempfile.TemporaryDirectory() as work:
        run(args.n, 10, work, args.imag)  # warm the driver / module load
        diffs = []
        for _ in range(args.repeat):
            a = run(args.n, args.n1, work, args.imag)
            b = run(args.n, args.n2, work, args.imag)
            diffs.append((b - a) / (args.n2 - args.n1))
    diffs.sort()
    per_step = diffs[len(diffs) // 2]
    print(json.dumps({"impl": "reference CUDA build (complex128, cuFFT)", "grid": [args.n] * 3,
                      "loop": "imaginary time (heavy ball)" if args.imag else "real-time RK4",
                      "steps_per_s": round(1.0 / per_step, 2), "ms_per_step": round(1e3 * per_step, 4),
                      "method": f"median over {args.repeat} of loop(niter={args.n2}) - loop(niter={args.n1}), "
                                "device-synchronised wall time of the reference's evolution loop",
                      "samples_ms_per_step": [round(1e3 * d, 4) for d in diffs]}))


if __name__ == "__main__":
    main()
