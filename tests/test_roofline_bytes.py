"""The per-kernel algorithmic byte model (pcom_b200.roofline) that bench.py's
roofline and the per-kernel GB/s report use."""
from pcom_b200.roofline import FIELDS, algorithmic_bytes


def test_barotropic_bytes_at_1_degree():
    # 120 substeps x 6 FP64 values (R/W ch, ub, vb) x 57,600 points + 30 static planes
    n2 = 360 * 160
    assert algorithmic_bytes("int_trop", 360, 160, 30, 120) == 8.0 * (120 * 6 * n2 + 30 * n2)
    # mixed: ub, vb in FP32, ch in FP64
    assert algorithmic_bytes("int_trop", 360, 160, 30, 120, mixed=True) == 120 * (16 + 16) * n2 + 8.0 * 30 * n2


def test_3d_fields_halve_on_the_mixed_path():
    for k, (f3, f2) in FIELDS.items():
        if k == "int_trop":
            continue
        d = algorithmic_bytes(k, 90, 40, 20, 120)
        m = algorithmic_bytes(k, 90, 40, 20, 120, mixed=True)
        n2 = 90 * 40
        assert d - m == 4.0 * f3 * n2 * 20, k
        assert m == 4.0 * f3 * n2 * 20 + 8.0 * f2 * n2, k


def test_unknown_kernel_moves_nothing():
    assert algorithmic_bytes("watchdog", 360, 160, 30, 120) == 0.0
