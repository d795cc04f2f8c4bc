#!/bin/sh
# Pins M(10^18) with the reference engine compiled from its own sources
# (make -C oracle ref).  The reference publishes no value for 10^18; this run is
# the only pin.  About 35 minutes on 8 cores.  Writes tests/golden/m1e18.json.
set -e
cd "$(dirname "$0")/../.."
T0=$(date +%s.%N)
OUT=$(oracle/_ref/bench_dr 1000000000000000000 8)
T1=$(date +%s.%N)
M=$(echo "$OUT" | sed -n 's/^M(1000000000000000000) = //p')
python - "$M" "$T0" "$T1" "$OUT" <<'PY'
import json, sys
m, t0, t1, out = sys.argv[1:5]
json.dump({"X": 10**18, "M": int(m), "source": "oracle/_ref/bench_dr 1000000000000000000 8 (reference engine, default env)",
           "wall_seconds": round(float(t1) - float(t0), 1), "threads": 8, "stdout": out.strip().splitlines()},
          open("tests/golden/m1e18.json", "w"), indent=1)
PY
