"""The half-pair kernel's job table (build_pair_jobs in
yukawamd_b200/csrc/yk_engine.cu, read through yk_pair_jobs; host arithmetic,
no GPU).  Every unit (R, C), C >= R, of the half-pair sum must be in exactly
one job, or a pair is lost or counted twice; jobs must respect the cap and
the guided sizes d <= max(1, W / 2P), W the work not yet handed out; and the
Si slots of a row must be 0 .. row_slots[R] - 1, each written once, because
k_combine sums exactly those.  The two-target table (build_pair_jobs2, read
through yk_pair_jobs2) must cover every unit of both rows of each block
pair exactly once and give both rows the same slots."""
import numpy as np
import pytest

from yukawamd_b200.engine import pair_jobs


@pytest.mark.parametrize("m,cap,ctas", [(1, 8, 888), (3, 4, 888), (32, 8, 888), (128, 4, 888),
                                        (432, 8, 740), (432, 4, 888), (700, 16, 296), (1024, 8, 888)])
def test_every_unit_once(m, cap, ctas):
    jobs, slots = pair_jobs(m, cap, ctas)
    R, C0, C1, s = jobs.T.astype(np.int64)
    assert np.all(C0 >= R) and np.all(C1 > C0) and np.all(C1 <= m)
    cover = np.zeros((m, m), dtype=np.int64)
    for r, a, b in zip(R, C0, C1):
        cover[r, a:b] += 1
    assert np.array_equal(cover, np.triu(np.ones((m, m), dtype=np.int64)))
    # slots of each row: 0 .. row_slots[R] - 1, each once
    for r in range(m):
        mine = np.sort(s[R == r])
        assert np.array_equal(mine, np.arange(slots[r]))


@pytest.mark.parametrize("m,cap,ctas", [(432, 8, 888), (1024, 16, 888), (128, 8, 148)])
def test_guided_sizes(m, cap, ctas):
    jobs, _ = pair_jobs(m, cap, ctas)
    size = (jobs[:, 2] - jobs[:, 1]).astype(np.int64)
    assert size.max() <= cap
    left = m * (m + 1) // 2 - np.concatenate(([0], np.cumsum(size)[:-1]))
    assert np.all(size <= np.maximum(1, left // (2 * ctas)))
    assert size[-1] == 1
    # the bulk goes out in capped jobs when there is enough work
    if m * (m + 1) // 2 > 4 * cap * ctas:
        assert size[0] == cap


def test_small_box_is_one_job():
    jobs, slots = pair_jobs(1, 8, 888)
    assert jobs.tolist() == [[0, 0, 1, 0]] and slots.tolist() == [1]


@pytest.mark.parametrize("m,cap,ctas", [(0, 8, 888), (4, 0, 888), (4, 8, 0)])
def test_bad_arguments(m, cap, ctas):
    with pytest.raises(ValueError):
        pair_jobs(m, cap, ctas)


@pytest.mark.parametrize("m,cap,ctas", [(1, 8, 592), (2, 8, 592), (3, 4, 592), (5, 1, 592), (33, 8, 592),
                                        (432, 8, 592), (432, 4, 592), (701, 16, 296)])
def test_two_target_jobs_cover_every_unit_once(m, cap, ctas):
    jobs, slots = pair_jobs(m, cap, ctas, targets_per_thread=2)
    R, C0, C1, s = jobs.T.astype(np.int64)
    assert np.all(R % 2 == 0) and np.all(C0 >= R) and np.all(C1 > C0) and np.all(C1 <= m)
    assert np.all(C1 - C0 <= cap)
    cover = np.zeros((m, m), dtype=np.int64)
    for r, a, b in zip(R, C0, C1):
        cover[r, a:b] += 1                      # block R: tiles C >= R
        if r + 1 < m:
            cover[r + 1, max(a, r + 1):b] += 1  # block R + 1: tiles C >= R + 1
    assert np.array_equal(cover, np.triu(np.ones((m, m), dtype=np.int64)))
    for r in range(0, m, 2):
        mine = np.sort(s[R == r])
        assert np.array_equal(mine, np.arange(slots[r]))
        if r + 1 < m:
            assert slots[r + 1] == slots[r]
