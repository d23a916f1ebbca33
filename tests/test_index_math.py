"""Integer shortcuts of the ICD kernel (timbir-python_b200/csrc/xtg_icd.cu),
checked exhaustively over the sizes the kernel accepts.

The neighbourhood staging divides k by Z + 2 as (k * m) >> 20 with
m = ceil(2^20 / (Z + 2)); work items hold at most 128 slices, and k runs
below 9 (Z + 2).  The product must be exact and fit in 32 bits."""


def test_multiply_shift_division_is_exact():
    for z in range(1, 129):
        d = z + 2
        m = ((1 << 20) + d - 1) // d
        for k in range(9 * d):
            assert k * m < 1 << 32
            assert (k * m) >> 20 == k // d, (z, k)


def test_entry_grouping_shifts():
    """Threads per footprint entry tlp = 2^lg >= tln = ceil(T / 4) rows
    groups; vg = tid >> lg, vgs = NT >> lg equal the divisions by tlp."""
    for nt in (64, 128, 256):
        for t in range(1, 129):
            tln = (t + 3) // 4
            lg = 0
            while (1 << lg) < tln:
                lg += 1
            tlp = 1 << lg
            if tlp > nt:
                continue
            assert nt >> lg == nt // tlp
            for tid in range(nt):
                assert tid >> lg == tid // tlp
