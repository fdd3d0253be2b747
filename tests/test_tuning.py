# SPDX-License-Identifier: Apache-2.0
"""The autotuner's record cache (no GPU): a cache file is read into the records, written back in
the same format, cleared; malformed or out-of-range lines are rejected with ValueError."""

from __future__ import annotations

import pytest


@pytest.fixture
def core():
    import eda

    c = eda._native.core()
    c.tuning_clear()
    yield c
    c.tuning_clear()


LINES = ["4 2 512 512 1 6 4 2 8 100.5 80.25", "8 1 2048 1 1 0 8 1 2 10 9"]


def test_cache_round_trip(core, tmp_path):
    p = tmp_path / "tune.txt"
    p.write_text("# a comment\n" + "\n".join(LINES) + "\n")
    core.tuning_load(str(p))
    dump = core.tuning_dump()
    rows = [ln for ln in dump.splitlines() if not ln.startswith("#")]
    assert sorted(r.split()[:9] for r in rows) == sorted(ln.split()[:9] for ln in LINES)
    q = tmp_path / "again.txt"
    q.write_text(dump)
    core.tuning_clear()
    assert [ln for ln in core.tuning_dump().splitlines() if not ln.startswith("#")] == []
    core.tuning_load(str(q))
    assert core.tuning_dump() == dump


@pytest.mark.parametrize("line", ["4 2 512", "3 2 512 512 1 6 4 2 8 1 1", "4 2 512 512 1 6 16 2 8 1 1",
                                  "4 2 512 512 1 6 4 9 8 1 1", "4 7 512 512 1 6 4 2 8 1 1"])
def test_bad_lines_are_rejected(core, tmp_path, line):
    p = tmp_path / "bad.txt"
    p.write_text(line + "\n")
    with pytest.raises(ValueError):
        core.tuning_load(str(p))


def test_missing_file_is_rejected(core, tmp_path):
    with pytest.raises(ValueError):
        core.tuning_load(str(tmp_path / "absent.txt"))
