"""Host side of the batch-plan autotuner (no GPU): the candidate plans it
times and the identity check every candidate must pass (a plan may only
change the time, never a path)."""
import torch

from orthoroute_b200.autotune import _candidates, _name, _same


def test_candidates_cover_both_kernels_on_lattices_only():
    lat = _candidates(1.5, True)
    gen = _candidates(1.5, False)
    assert {c["impl"] for c in lat} == {0, 1} and {c["impl"] for c in gen} == {0}
    assert sorted(c["tile_w"] for c in lat if c["impl"] == 1) == [16, 32]
    assert sorted({c["delta"] for c in gen}) == [0.75, 1.5, 3.0, 6.0]
    assert len({_name(c) for c in lat}) == len(lat)  # distinct names in the tuning table


def test_same_compares_lengths_and_paths_only_up_to_each_length():
    nodes = torch.tensor([[1, 2, 3, 9], [4, 5, 0, 0]], dtype=torch.int32)
    lens = torch.tensor([3, 2], dtype=torch.int32)
    ref = (nodes, None, lens)
    other = nodes.clone()
    other[0, 3] = 7  # past the path's end: ignored
    other[1, 2:] = 8
    assert _same(ref, (other, None, lens.clone()), 2)
    other[1, 1] = 6  # inside the second path
    assert not _same(ref, (other, None, lens.clone()), 2)
    assert not _same(ref, (nodes, None, torch.tensor([3, 0], dtype=torch.int32)), 2)
