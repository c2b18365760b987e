"""The algorithmic bytes model the roofline figures are computed from."""
import bytes_model as bm


def test_plain_form_counts_accesses_at_eight_bytes():
    assert bm.bytes_per_cell_iteration(False, 0) == 8 * 108
    assert bm.bytes_per_cell_iteration(True, 200) == 8 * (218 + 12 * 200)


def test_mixed_form_counts_inner_iterations_at_four_bytes():
    b = bm.bytes_per_cell_iteration_mixed(True, 16)
    assert b == 8 * (218 + 21) + 4 * 60 * 16
    # the benchmark pair: the mixed form's launch moves ~3.6x fewer bytes
    assert 3.5 < bm.bytes_per_cell_iteration(True, 200) / b < 3.8
