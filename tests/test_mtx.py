"""Matrix Market ingest (rak_read_mtx): the reference driver's reading rules (readMtxOmpW +
symmetrizeOmpU), checked on hand-made files with known CSRs and, where the reference's CPU code is
built (oracle/_ref), against the reference's own reader on the same files."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl


def write(path, text):
    path.write_text(text)
    return str(path)


def csr_of(g):
    return [list(g.targets[g.offsets[u]:g.offsets[u + 1]]) for u in range(g.n)]


def test_general_pattern_symmetrized(tmp_path):
    p = write(tmp_path / "a.mtx", "%%MatrixMarket matrix coordinate pattern general\n% a comment\n"
                                  "4 4 4\n1 2\n2 3\n3 1\n4 4\n")
    g = rl.read_mtx(p, weighted=False, symmetrize=True)
    assert g.n == 4 and g.weights is None
    assert csr_of(g) == [[1, 2], [0, 2], [0, 1], [3]]
    g2 = rl.read_mtx(p, weighted=False, symmetrize=False)
    assert csr_of(g2) == [[1], [2], [0], [3]]


def test_symmetric_real_zero_weight_and_diagonal(tmp_path):
    p = write(tmp_path / "b.mtx", "%%MatrixMarket matrix coordinate real symmetric\n"
                                  "3 3 4\n2 1 2.5\n3 1 0\n3 3 4.0\n3 2 1e-1\n")
    g = rl.read_mtx(p, weighted=True)
    assert csr_of(g) == [[1, 2], [0, 2], [0, 1, 2]]
    w = [list(g.weights[g.offsets[u]:g.offsets[u + 1]]) for u in range(g.n)]
    assert w == [[2.5, 1.0], [2.5, np.float32(0.1)], [1.0, np.float32(0.1), 4.0]]   # 0 reads as 1


def test_skew_symmetric_duplicates_and_rectangular(tmp_path):
    p = write(tmp_path / "c.mtx", "%%MatrixMarket matrix coordinate integer skew-symmetric\n"
                                  "2 5 3\n2 1 3\n2 1 3\n5 2 7\n")
    g = rl.read_mtx(p, weighted=True)
    assert g.n == 5
    assert csr_of(g) == [[1], [0, 4], [], [], [1]]
    assert list(g.weights) == [3, 3, 7, 7]


def test_repeated_pair_keeps_last(tmp_path):
    p = write(tmp_path / "d.mtx", "%%MatrixMarket matrix coordinate real general\n3 3 3\n1 2 5\n1 2 6\n2 1 9\n")
    g = rl.read_mtx(p, weighted=True, symmetrize=False)
    assert csr_of(g) == [[1], [0], []] and list(g.weights) == [6, 9]


def test_not_coordinate_is_empty(tmp_path):
    p = write(tmp_path / "e.mtx", "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    g = rl.read_mtx(p)
    assert g.n == 0 and g.m == 0


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(rl.RakError):
        rl.read_mtx(str(tmp_path / "none.mtx"))


@pytest.mark.skipif(not orc.have_ref_cpu(), reason="reference CPU build (oracle/_ref) not present")
@pytest.mark.parametrize("symmetry,weighted,symmetrize", [("general", True, True), ("general", False, True),
                                                          ("general", True, False), ("symmetric", True, True),
                                                          ("symmetric", False, False)])
def test_matches_reference_reader(tmp_path, symmetry, weighted, symmetrize):
    rng = np.random.default_rng(hash((symmetry, weighted, symmetrize)) & 0xFFFF)
    n, e = 2000, 12000
    u = rng.integers(1, n + 1, e)
    v = rng.integers(1, n + 1, e)
    if symmetry == "symmetric":
        u, v = np.maximum(u, v), np.minimum(u, v)          # lower triangle, as such files store it
    # a repeated pair always carries the same weight here: the reference keeps an arbitrary one of
    # several (unstable sort), this library the last
    w = ((u * 7919 + v * 104729) % 1000) / 100.0
    lines = "\n".join(f"{a} {b} {c:g}" if weighted else f"{a} {b}" for a, b, c in zip(u, v, w))
    field = "real" if weighted else "pattern"
    p = write(tmp_path / "r.mtx", f"%%MatrixMarket matrix coordinate {field} {symmetry}\n{n} {n} {e}\n{lines}\n")
    g = rl.read_mtx(p, weighted=weighted, symmetrize=symmetrize)
    off, tgt, wt = orc.ref_read_mtx(p, weighted=weighted, symmetrize=symmetrize)
    np.testing.assert_array_equal(g.offsets, off)
    np.testing.assert_array_equal(g.targets, tgt)
    if weighted:
        np.testing.assert_array_equal(g.weights, wt)
    else:
        assert g.weights is None
