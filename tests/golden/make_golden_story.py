"""Golden vectors of the snapshot reader: the reference's own get_dyn
(oracle/_ref/story_ref, built from the reference sources by
oracle/build_ref.py) run on two seeded story texts, every value kept
exactly.  Writes tests/golden/story_*.npz (text and arrays).

Usage: python tests/golden/make_golden_story.py  (needs oracle/_ref built).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import ref_story  # noqa: E402
from story_texts import VARIANTS, flat_text, hierarchy_text  # noqa: E402

CASES = {
    "story_flat_n64": lambda: flat_text(64, 5),
    "story_hierarchy_3roots": lambda: hierarchy_text(11, roots=3, leaves_per_root=12),
}
# one fixture per corner-case text
for _k, _t in sorted(VARIANTS.items()):
    CASES["story_variant_" + _k.replace(" ", "_").replace("-", "_")] = (lambda t: (lambda: t))(_t)


def main():
    for name, make in CASES.items():
        text = make()
        r = ref_story(text)
        if r is None:
            raise SystemExit("oracle/_ref/story_ref not built")
        np.savez_compressed(os.path.join(HERE, name + ".npz"), text=np.frombuffer(text, np.uint8),
                            parent=r.parent, index=r.index, mass=r.mass, pos=r.pos, vel=r.vel,
                            leaves_pos=r.leaves_pos, leaves_vel=r.leaves_vel, system_time=r.system_time)
        print(name, r.parent.size, "nodes")


if __name__ == "__main__":
    main()
