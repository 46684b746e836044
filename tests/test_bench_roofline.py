"""bench.py's algorithmic FP64 work per PML element, the numerator of the
reported roofline: the full product of k_pml_mma / k_pml_ws (4 flops per
staged row and matrix entry, 3 rows per curl point, 6 per mass point with
the cross terms) and the triangle-plus-cross-part count of k_pml_sym."""

from __future__ import annotations

import bench


def test_full_product_p3():
    # nd = 45, 11 curl points, 24 mass points: K = 3 * 11 + 6 * 24 = 177 rows
    assert bench.pml_flops(1, 45, 11, 24, True, 0) == 4 * 177 * 45 * 45 == 1_433_700
    assert bench.pml_flops(1, 45, 11, 24, True, 1) == 1_433_700
    # without the cross terms the mass rule stages 3 rows a point
    assert bench.pml_flops(1, 45, 11, 24, False, 0) == 4 * (33 + 72) * 2025


def test_symmetric_split_p3():
    tri = 45 * 46 // 2
    want = 4 * (3 * 35 * tri + 3 * 24 * 45 * 45)
    assert bench.pml_flops(1, 45, 11, 24, True, 2) == want == 1_017_900
    assert bench.pml_flops(1, 45, 11, 24, False, 2) == 4 * 3 * 35 * tri


def test_scales_with_the_element_count():
    assert bench.pml_flops(13_608, 45, 11, 24, True, 1) == 13_608 * 1_433_700
