#!/usr/bin/env python3
"""Generate golden fixtures by running the REFERENCE's own CUDA build on a GPU.

Binaries come from oracle/ref.mk (built from the reference sources):
  oracle/_ref/gpe_ref_trace  reference sources + test plugins that fill
                             d_h_params from quench_* keys and log PARS
  oracle/_ref/gpe_ref        the stock reference binary (its own plugins)
Each case in tests/golden/inputs/ is run in order (real-time cases read the
psi_final.wdat of the imaginary-time case before them) and packed as
tests/golden/<case>.npz: the input text, psi_init / vext / psi_final arrays,
the PARS trace, and for stock cases status.out, info.wtxt and psi.wdat frames.

Usage (on a GPU host):  python tests/golden/make_golden.py --out DIR
"""
import argparse
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
import golden_util as gu  # noqa: E402
REF_TRACE = os.path.join(ROOT, "oracle", "_ref", "gpe_ref_trace")
REF_STOCK = os.path.join(ROOT, "oracle", "_ref", "gpe_ref")

# (case, binary, number of components)
CASES = [
    ("g_hb_bec", REF_TRACE, 1),
    ("g_hb_conv", REF_TRACE, 1),
    ("g_rt_quench", REF_TRACE, 1),
    ("g_hb_bec2", REF_TRACE, 2),
    ("g_rt_bec2", REF_TRACE, 2),
    ("g_hb_template", REF_TRACE, 1),
    ("g_stock_2d", REF_STOCK, 1),
    ("g_stock_rt", REF_STOCK, 1),
    ("g_stock_rot", REF_STOCK, 1),
    ("g_stock_rot_rt", REF_STOCK, 1),
    ("g_cfg1_hb64", REF_TRACE, 1),
]


def read_c128(fn):
    return np.fromfile(fn, dtype=np.complex128) if os.path.exists(fn) else np.zeros(0, np.complex128)


def parse_trace(fn):
    rows = []
    if not os.path.exists(fn):
        return np.zeros((0, 0))
    for line in open(fn):
        f = line.split()
        if not f or f[0] == "end":
            continue
        tag = {"im": 0.0, "conv": 1.0, "re": 2.0}[f[0]]
        rows.append([tag] + [float(x) for x in f[1:]])
    return np.array(rows)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--pack-into", default=None, help="directory for the .npz fixtures (default: --out)")
    ap.add_argument("--only", nargs="*", default=None,
                    help="cases to run (a real-time case needs its imaginary-time case in the same call)")
    args = ap.parse_args()
    work = os.path.abspath(os.path.join(args.out, "run"))
    os.makedirs(work, exist_ok=True)
    pack = os.path.abspath(args.pack_into or args.out)
    os.makedirs(pack, exist_ok=True)
    for case, binary, nc in CASES:
        if args.only is not None and case not in args.only:
            continue
        src = open(os.path.join(HERE, "inputs", case + ".txt")).read()
        inp = os.path.join(work, case + ".txt")
        with open(inp, "w") as f:
            f.write(src.replace("@OUT@", work + "/"))
        generated = None
        if case in gu.GENERATED:
            # the trap and the seeded initial state, as the .wdat files the input reads
            _, o = gu.params_dump(src, work)
            psi, V = gu.cfg1_inputs(o)
            keys = gu.keys(src.replace("@OUT@", work + "/"))
            psi.astype(np.complex128).tofile(keys["inprefix"].strip('"') + "psi_final.wdat")
            V.astype(np.complex128).tofile(keys["vprefix"].strip('"') + "vext.wdat")
            generated = gu.input_checksums(psi, V)
        r = subprocess.run([binary, inp], capture_output=True, text=True, timeout=600)
        with open(os.path.join(work, case + ".log"), "w") as f:
            f.write(r.stdout + "\n---stderr---\n" + r.stderr)
        if r.returncode != 0:
            print(f"{case}: reference exited {r.returncode}", file=sys.stderr)
            sys.exit(1)
        pre = os.path.join(work, case + "_")
        d = {"input": np.array(src), "ncomp": np.array(nc), "stdout": np.array(r.stdout)}
        if generated is not None:
            # the reference wrote back the state and trap it read
            for name, arr in (("psi_init.wdat", psi), ("vext.wdat", V)):
                got = read_c128(pre + name)
                if got.size and not np.array_equal(got, arr):
                    print(f"{case}: {name} differs from the generated input", file=sys.stderr)
                    sys.exit(1)
            d.update(generated)
            d["psi_final"] = read_c128(pre + "psi_final.wdat")
        elif nc == 1:
            d["psi_init"] = read_c128(pre + "psi_init.wdat")
            d["vext"] = read_c128(pre + "vext.wdat")
            d["psi_final"] = read_c128(pre + "psi_final.wdat")
        else:
            for c in (1, 2):
                d[f"psi_init{c}"] = read_c128(pre + f"{c}psi_init.wdat")
                d[f"vext{c}"] = read_c128(pre + f"{c}vext.wdat")
                d[f"psi_final{c}"] = read_c128(pre + f"{c}psi_final.wdat")
        d["trace"] = parse_trace(pre + "trace.txt")
        for name in ("status.out", "info.wtxt"):
            fn = pre + name
            if os.path.exists(fn):
                d[name.replace(".", "_")] = np.array(open(fn).read())
        if os.path.exists(pre + "psi.wdat"):
            d["psi_frames"] = read_c128(pre + "psi.wdat")
        np.savez_compressed(os.path.join(pack, case + ".npz"), **d)
        print(f"{case}: ok ({len(d['trace'])} trace rows)")


if __name__ == "__main__":
    main()
