"""CPU: the seeded instance draw of the batched uneven workload matches its committed
manifest, and covers the stated ranges."""
from fr_sdg_b200.batch import SIZES, draw_instances, load_manifest


def test_manifest_reproduces():
    assert draw_instances() == load_manifest()


def test_draw_ranges():
    sp = load_manifest()
    assert len(sp) == 512
    assert {s.n_elems for s in sp} == set(SIZES) and {s.p for s in sp} == {2, 3, 4, 5, 6}
    for s in sp:
        if s.gas == "ideal":
            assert 1.3 <= s.gamma <= 1.67 and s.vdw_a == s.vdw_b == 0.0
        else:
            assert s.gamma == 1.4 and 0.01 <= s.vdw_a <= 0.1 and 0.01 <= s.vdw_b <= 0.05
        assert 0.3 <= s.r0 <= 0.5 and 0.05 <= s.p_out <= 0.2
    nodes = sum(s.n_elems ** 2 * (s.p + 1) ** 2 for s in sp)
    assert 80e6 < nodes < 100e6
