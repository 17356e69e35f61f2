"""One story-reader workload for profiling: a flat N-body snapshot in the
reference's output format (root + N leaves, "%.18g"), resident in device
memory, parsed --reps times with check_and_correct_node and --reps times
raw.  Prints the median wall time of each.

    python -m starlab_b200.profile_story --n 262144 --reps 3
"""
import argparse
import statistics
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=11)
    a = ap.parse_args(argv)
    import torch
    from starlab_b200 import ics
    from starlab_b200.story import StoryReader, format_story
    m = ics.salpeter_masses(a.n, a.seed)
    _, x, v = ics.plummer(a.n, a.seed + 1, masses=m)
    text = format_story(m, x + 1e-3, v - 5e-4)
    d = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    rd = StoryReader()
    for raw in (False, True):
        ts = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            info = rd.parse_device(d.data_ptr(), d.numel(), raw=raw)
            ts.append(time.perf_counter() - t0)
        print("raw=%d n=%d bytes=%d nodes=%d median %.3f ms" % (raw, a.n, len(text), info.n_nodes,
                                                                 1e3 * statistics.median(ts)))
    rd.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
