"""Reference digests of the full-size benchmark clouds, made by the reference itself.

The reference (compiled from its own sources into oracle/_ref by oracle/build_ref.sh)
compresses and decompresses each seeded cloud in every variant of its workload; this
script records, per variant, the SHA-256 and length of the reference's zstd frame, of its
pre-zstd container and of the points its decompressor returns, plus the SHA-256 of the
generated input (so a checker can first confirm it regenerated the same cloud).  The GPU
path is checked against these digests by bench.py (64M-point terrain, 175M-point spheres)
and by tests/test_gpu_digests.py (8M-point terrain), on machines without the reference.

    python tests/golden/make_ref_digests.py --workload terrain --points 8000000
    python tests/golden/make_ref_digests.py --workload terrain --points 64000000 --jobs 3
    python tests/golden/make_ref_digests.py --workload spheres --points 175000000 --jobs 1

Each variant runs in its own spawned process (the reference is single-threaded); --jobs
bounds how many run at once (a 64M-point variant holds about 10 GB).  Results are merged
into tests/golden/ref_digests.json.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "ref_digests.json")

# (quantizer, l2, hilbert, rle) per workload, in the order bench.py runs them
WORKLOADS = {
    "terrain": [("to", 0.001, 1, 1), ("to", 0.01, 1, 1), ("to", 0.1, 1, 1),
                ("cube", 0.001, 1, 1), ("cube", 0.01, 1, 1), ("cube", 0.1, 1, 1)],
    "spheres": [("to", 0.5, 0, 0), ("to", 0.5, 0, 1)],
}


def synthetic():
    """The seeded generators, loaded from their file (the package itself is not imported)."""
    spec = importlib.util.spec_from_file_location("xnyz_synthetic", os.path.join(ROOT, "xnyzip_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cloud(workload: str, n: int, seed: int):
    S = synthetic()
    return S.spheres(n, 200_000, seed) if workload == "spheres" else S.terrain(n, seed)


def variant_name(q, l2, hil, rle):
    return f"{q}_{l2}" + ("" if (hil, rle) == (1, 1) else f"_{'h' if hil else 'z'}_{'rle' if rle else 'normal'}")


def sha(b) -> str:
    return hashlib.sha256(memoryview(b).cast("B")).hexdigest()


def run_variant(workload: str, n: int, seed: int, v):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    q, l2, hil, rle = v
    x = cloud(workload, n, seed)
    ref = Reference()
    ref.quiet(True)
    t0 = time.time()
    frame = ref.compress(x, q, l2, hil, rle)
    container = ref.unzstd(frame)
    pts = ref.decompress(frame, q, l2, rle)
    ref.quiet(False)
    return variant_name(*v), {
        "frame_sha256": sha(frame), "frame_bytes": len(frame),
        "container_sha256": sha(container), "container_bytes": len(container),
        "points_sha256": sha(pts.tobytes()), "points_out": int(pts.shape[0]),
        "reference_s": round(time.time() - t0, 1),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="terrain", choices=sorted(WORKLOADS))
    ap.add_argument("--points", type=int, required=True)
    ap.add_argument("--seed", type=int, default=0, help="0: the bench's seed (terrain 1, spheres 2)")
    ap.add_argument("--jobs", type=int, default=1)
    args = ap.parse_args()
    seed = args.seed or (2 if args.workload == "spheres" else 1)
    key = f"{args.workload}_{args.points}_seed{seed}"
    x = cloud(args.workload, args.points, seed)
    entry = {"workload": args.workload, "points": args.points, "seed": seed, "input_sha256": sha(x.tobytes()),
             "direct_threshold": 1024, "variants": {}}
    del x
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.jobs) as pool:
        res = pool.starmap(run_variant, [(args.workload, args.points, seed, v) for v in WORKLOADS[args.workload]])
    for name, d in res:
        entry["variants"][name] = d
        print(name, d, flush=True)
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data[key] = entry
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", key, "to", OUT)


if __name__ == "__main__":
    main()
