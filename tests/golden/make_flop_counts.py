"""Per-photon operation counts of the benchmark workload, from one
instrumented run of the CPU oracle (oracle/merlict_oracle.c counts every
bounding-sphere test, leaf transform, cap quadratic, cap bound, plane test,
reflection, Fresnel step, time-of-flight segment and table look-up).

bench.py weights these counts with the FLOP cost of each operation in the
reference's own code to state the work per photon.

    python tests/golden/make_flop_counts.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import bench  # noqa: E402
from merlict_development_kit_b200 import factories as F  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

N = 200_000


def main():
    flat = F.light_field_telescope(**bench.SCENE).flatten()
    ph = bench.make_photons(N, 777)
    status, out, counts = Oracle().propagate(flat, ph, bench.MAX_INTERACTIONS, seed=5)
    assert status == 0
    per = {k: v / N for k, v in counts.items()}
    doc = {"workload": bench.WORKLOAD, "scene": bench.scene_config_name(), "photons": N,
           "seed": 5, "max_interactions": bench.MAX_INTERACTIONS, "per_photon": per}
    with open(os.path.join(HERE, "flop_counts.json"), "w") as f:
        json.dump(doc, f, indent=1)
    flops = sum(bench.FLOP_WEIGHTS[k] * per.get(k, 0.0) for k in bench.FLOP_WEIGHTS)
    print(json.dumps(per, indent=1), "\nFLOP per photon", flops)


if __name__ == "__main__":
    main()
