"""bench.py's claims that need no GPU: the launch count it reports as
`gpu_launches` agrees with the ncu launch lists committed under profiles/
(two steps of each form per list)."""
from __future__ import annotations

import importlib.util
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _launches(profile: str, section: str | None = None) -> dict:
    text = open(os.path.join(ROOT, "profiles", profile)).read()
    if section:  # the lists under a "# <section>" heading, up to the next one
        text = text.split(f"# {section}\n", 1)[1].split("\n# ", 1)[0]
    found = re.findall(r"## (plain|chosen) form: (\d+) launches", text)
    assert len(found) == 2, found
    return {k: int(v) for k, v in found}


def test_launch_count_matches_the_committed_launch_list():
    b = _bench()
    counts = _launches("launches_step_impact_1e6.md")  # chosen form captured with 8 online Adam steps
    assert counts["plain"] == 2 * b.launches_per_step(b.DEPTH, False)
    assert counts["chosen"] == 2 * b.launches_per_step(b.DEPTH, True, 8)


def test_small_impact_launch_lists_have_the_same_structure():
    # the 2e4 lists were captured with the bench's default refresh depth
    b = _bench()
    counts = _launches("launches_step_impact_2e4_coarse_tiles.md", "coarse tiles on")
    assert counts["plain"] == 2 * b.launches_per_step(b.DEPTH, False)
    assert counts["chosen"] == 2 * b.launches_per_step(b.DEPTH, True, 4)
    # without the coarse tiles each of the two tile passes skips its coarse
    # tile list and coarse pass
    off = _launches("launches_step_impact_2e4_coarse_tiles.md", "coarse tiles off")
    assert counts["plain"] - off["plain"] == 2 * 4 and counts["chosen"] - off["chosen"] == 2 * 4


def test_ensemble_instances_run_no_seed_kernels():
    b = _bench()
    assert b.launches_per_step(b.DEPTH, True, seed=False) == b.launches_per_step(b.DEPTH, True) - 3
