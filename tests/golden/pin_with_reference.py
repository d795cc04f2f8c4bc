"""Pin M(X) for an X the reference publishes no value for, by running the
reference engine compiled from its own sources (oracle/_ref/bench_dr):

    python tests/golden/pin_with_reference.py 30000000000000000 [threads]

Writes tests/golden/m<X>.json with the value, the command and its wall time.
"""
import json
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    X = int(sys.argv[1])
    threads = sys.argv[2] if len(sys.argv) > 2 else "8"
    cmd = [os.path.join(ROOT, "oracle", "_ref", "bench_dr"), str(X), threads]
    t0 = time.time()
    out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
    dt = time.time() - t0
    M = int(out.split(f"M({X}) = ")[1].split()[0])
    rec = {"X": X, "M": M, "source": f"oracle/_ref/bench_dr {X} {threads} (reference engine, default env)",
           "wall_seconds": round(dt, 1), "threads": int(threads), "stdout": out.strip().splitlines()}
    with open(os.path.join(HERE, f"m{X}.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(rec)


if __name__ == "__main__":
    main()
