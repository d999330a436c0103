"""The swizzled shared-memory layout of the TMA-fed Horner kernel
(csrc/batch_tma.cuh), restated on the CPU: every DMMA fragment load of the
m16n8k8 .f64 layout, through the kernel's permuted fragment rows and columns
and its precomputed offsets (with the XOR shortcuts it applies per k-step),
reads the element the layout asks for, and every half-warp load covers 16
distinct 8-byte bank slots (no bank conflict), for the k-major coupling tile
(D_{L-1}^T), the m-major one (D_L) and the state tile alike."""

FRAG_ROW = 0x9A56B874DE12FC30   # nibble g: the tile row of fragment row g


def frag_row(g):
    return (FRAG_ROW >> (4 * g)) & 15


def frag_col(nb, g):
    return 4 * nb + (g & 1) + 8 * ((g >> 1) & 1) + 2 * (g >> 2)


def swz(r, c):
    """Offset (doubles) of line r, column c of a 128-byte-wide box stored
    with the 128-byte TMA swizzle (16-byte chunk c/2 of line r at c/2 ^ r%8)."""
    return r * 16 + ((((c >> 1) ^ (r & 7))) << 1) + (c & 1)


def addr_p(k, m):      # k-major tile: 16-row groups of m, 32 lines of k each
    return (m >> 4) * 512 + swz(k, m & 15)


def addr_q(m, k):      # m-major tile: 16-column groups of k, 64 lines of m each
    return (k >> 4) * 1024 + swz(m, k & 15)


def addr_b(k, n):      # state tile: 16-column groups of n, 32 lines of k each
    return (n >> 4) * 512 + swz(k, n & 15)


def bank_slot(off):
    return (off * 8 % 128) // 8


def test_permutations_are_permutations():
    assert sorted(frag_row(g) for g in range(16)) == list(range(16))
    assert sorted(frag_col(nb, g) for nb in (0, 1) for g in range(8)) == list(range(16))
    # a fragment column pair (2t, 2t+1) is one pulse: adjacent, even first
    for nb in (0, 1):
        for t in range(4):
            x, y = frag_col(nb, 2 * t), frag_col(nb, 2 * t + 1)
            assert x % 2 == 0 and y == x + 1
            assert x == 4 * nb + 2 * (t >> 1) + 8 * (t & 1)


def test_coupling_fragments_read_the_right_elements_without_conflicts():
    for mtile in range(4):
        for ks in range(4):
            for reg in range(4):          # a0 a1 a2 a3
                for half in range(2):
                    sp, sq = set(), set()
                    for lane in range(16 * half, 16 * half + 16):
                        g, t = lane >> 2, lane & 3
                        gl = g + (8 if reg in (1, 3) else 0)
                        k = ks * 8 + t + (4 if reg >= 2 else 0)
                        m = 16 * mtile + frag_row(gl)
                        # k-major: offset at k-step 0, + ks*128, k+4 as (^8)+64
                        o = mtile * 512 + swz(t, frag_row(gl))
                        o = ((o ^ 8) + 64 if reg >= 2 else o) + ks * 128
                        assert o == addr_p(k, m)
                        sp.add(bank_slot(o))
                        # m-major: box ks/2, odd ks as ^8, k+4 as ^4
                        q = swz(16 * mtile + frag_row(gl), t)
                        q = q ^ 4 if reg >= 2 else q
                        q = (q ^ 8 if ks & 1 else q) + (ks >> 1) * 1024
                        assert q == addr_q(m, k)
                        sq.add(bank_slot(q))
                    assert len(sp) == 16 and len(sq) == 16


def test_state_fragments_read_the_right_elements_without_conflicts():
    for j in range(8):                    # 8-column n-tiles of a 64-column tile
        for ks in range(4):
            for reg in range(2):          # b0 b1
                for half in range(2):
                    sb = set()
                    for lane in range(16 * half, 16 * half + 16):
                        g, t = lane >> 2, lane & 3
                        n = 16 * (j >> 1) + frag_col(j & 1, g)
                        k = ks * 8 + t + 4 * reg
                        o = (j >> 1) * 512 + swz(t, frag_col(j & 1, g))
                        o = ((o ^ 8) + 64 if reg else o) + ks * 128
                        assert o == addr_b(k, n)
                        sb.add(bank_slot(o))
                    assert len(sb) == 16
