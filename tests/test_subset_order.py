"""Sub-iteration -> subset order (IterativeReconstruction::get_subset_num), in order and uniformly randomised."""
from stir_b200.subsets import SubsetOrder


def test_in_order_with_start_subset():
    o = SubsetOrder(6, start_subset_num=2)
    assert [o(k) for k in range(1, 9)] == [2, 3, 4, 5, 0, 1, 2, 3]


def test_randomised_order_is_a_permutation_per_iteration():
    o = SubsetOrder(21, uniformly_randomise_subset_order=True, seed=7)
    seq = [o(k) for k in range(1, 3 * 21 + 1)]
    for it in range(3):
        assert sorted(seq[21 * it:21 * (it + 1)]) == list(range(21))
    assert seq[:21] != list(range(21))
    assert seq[:21] != seq[21:42]  # a new permutation every full iteration


def test_randomised_order_repeats_with_the_seed_and_per_subiteration():
    a = SubsetOrder(6, uniformly_randomise_subset_order=True, seed=3)
    b = SubsetOrder(6, uniformly_randomise_subset_order=True, seed=3)
    # asking twice for the same sub-iteration does not draw a new permutation
    sa = [(a(k), a(k)) for k in range(1, 13)]
    assert all(x == y for x, y in sa)
    assert [x for x, _ in sa] == [b(k) for k in range(1, 13)]
