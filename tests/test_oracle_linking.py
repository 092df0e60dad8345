"""Known-answer cases for the linker restatement (src/linking.rs).

The reference has no tests and its Rust cannot be built here, so these
cases are derived by hand from linking.rs: optimal (not greedy) subnet
assignment with null cost search_range^2, strict `<` on distances and on
score improvement, new ids in destination order, the memory ring, the
TooDenseToLink load guard, and the FrameSubsetter quirks.
"""
import numpy as np
import pytest


def fyx(rows):
    return np.array(rows, np.float32).reshape(-1, 3)


def test_simple_two_particles(oracle):
    ids = oracle.link(fyx([[0, 0, 0], [0, 10, 10], [1, 0.5, 0.2], [1, 10.3, 9.9]]), 2.0, 0)
    assert ids.tolist() == [0, 1, 0, 1]


def test_optimal_beats_greedy(oracle):
    # sources at x=0, x=2; dests at x=1.1 (closer to source 1) and x=3.0.
    # greedy: d0<-s1 (0.81) + d1 null (6.25) = 7.06; optimal: d0<-s0 (1.21) + d1<-s1 (1.0)
    ids = oracle.link(fyx([[0, 0, 0], [0, 0, 2], [1, 0, 1.1], [1, 0, 3.0]]), 2.5, 0)
    assert ids.tolist() == [0, 1, 0, 1]


def test_new_particle_and_order(oracle):
    # dest order decides new ids: the unmatched dests get 2 then 3
    ids = oracle.link(fyx([[0, 0, 0], [0, 50, 50], [1, 30, 30], [1, 0.1, 0.1], [1, 80, 80], [1, 50, 50.2]]),
                      3.0, 0)
    assert ids.tolist() == [0, 1, 2, 0, 3, 1]


def test_distance_is_strict(oracle):
    # exactly search_range away is not a neighbour (dist^2 < r^2)
    ids = oracle.link(fyx([[0, 0, 0], [1, 0, 2.0]]), 2.0, 0)
    assert ids.tolist() == [0, 1]


def test_memory_relinks_after_gap(oracle):
    rows = [[0, 5, 5], [0, 40, 40], [1, 40.5, 40], [2, 5.3, 5.1], [2, 40.2, 40.4]]
    assert oracle.link(fyx(rows), 2.0, 0).tolist() == [0, 1, 1, 2, 1]
    assert oracle.link(fyx(rows), 2.0, 1).tolist() == [0, 1, 1, 0, 1]


def test_memory_expires(oracle):
    rows = [[0, 5, 5], [0, 40, 40], [1, 40.5, 40], [2, 40.2, 40.4], [3, 5.3, 5.1]]
    assert oracle.link(fyx(rows), 2.0, 1).tolist() == [0, 1, 1, 1, 2]
    assert oracle.link(fyx(rows), 2.0, 2).tolist() == [0, 1, 1, 1, 0]


def test_too_dense_to_link(oracle):
    rng = np.random.default_rng(0)
    n = 72  # one subnet with load 72*72 = 5184 > 5000
    a = rng.uniform(0, 1, (n, 2))
    b = rng.uniform(0, 1, (n, 2))
    rows = np.r_[np.c_[np.zeros(n), a], np.c_[np.ones(n), b]]
    with pytest.raises(oracle.OracleError) as e:
        oracle.link(rows, 5.0, 0)
    assert e.value.code == 8  # GT_ERR_TOO_DENSE_TO_LINK
    n = 70  # load 4900 passes the guard (the search itself is pruned quickly)
    rows = np.r_[np.c_[np.zeros(n), a[:n]], np.c_[np.ones(n), a[:n] + 1e-3]]
    ids = oracle.link(rows, 0.01, 0)
    assert ids[n:].tolist() == list(range(n))


def test_single_dest_multi_source_subnet(oracle):
    # one dest between two sources: the closer source wins, the other leaves
    ids = oracle.link(fyx([[0, 0, 0], [0, 0, 3], [1, 0, 1.2]]), 2.0, 0)
    assert ids.tolist() == [0, 1, 0]


def test_tie_keeps_first_enumerated(oracle):
    # both assignments cost the same; strict `<` keeps the first found
    # (dest 0 takes its first-listed source, source 0)
    ids = oracle.link(fyx([[0, 0, 0], [0, 0, 2], [1, 0, 1], [1, 0, 3]]), 1.5, 0)
    assert ids.tolist() == [0, 1, 0, 1]


def test_unsorted_frames_raise(oracle):
    with pytest.raises(oracle.OracleError) as e:
        oracle.link(fyx([[1, 0, 0], [0, 1, 1]]), 2.0, 0)
    assert e.value.code == 4  # NonSortedCharacterization


def test_frames_may_start_late_and_skip(oracle):
    # a leading empty frame 0 is linked first; gaps in frame numbers are not
    # counted by the linker (it sees consecutive groups)
    ids = oracle.link(fyx([[3, 1, 1], [7, 1.5, 1.0]]), 2.0, 0)
    assert ids.tolist() == [0, 0]


def test_connect(oracle):
    a = fyx([[0, 0, 0], [0, 10, 10], [2, 5, 5]])
    b = fyx([[0, 0.1, 0.0], [1, 3, 3], [2, 20, 20]])
    ia, ib = oracle.connect(a, b, 1.0)
    # frame 0: a0<->b0 connected, a1 alone; frame 1 only in b; frame 2 no match
    assert ia[0] == ib[0]
    assert len(set(ia.tolist()) | set(ib.tolist())) == 5
