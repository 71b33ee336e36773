"""Host-side logic of the drop-in modules (no GPU): VCF and population-file readers,
biallelic filters, statistic names/specs, chunk sizing, genetic-map helpers."""
import json
import os

import numpy as np

from oracle import ld_oracle as O
from pg_gpu_b200 import genotype_matrix, haplotype_matrix, ld_pipeline, moments_ld

VCF = """##fileformat=VCFv4.2
#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\ts0\ts1\ts2
1\t10\t.\tA\tT\t.\tPASS\t.\tGT\t0|1\t1|1\t0|0
1\t25\t.\tA\tC\t.\tPASS\t.\tGT\t0|0\t0|0\t0|0
1\t40\t.\tG\tA\t.\tPASS\t.\tGT\t.|1\t0|1\t1|0
1\t55\t.\tG\tA,T\t.\tPASS\t.\tGT\t0|2\t0|1\t1|0
1\t90\t.\tC\tG\t.\tPASS\t.\tGT\t1|0:30\t0|1:20\t1|1:10
"""


def test_vcf_reader_layout_and_filter(tmp_path):
    p = tmp_path / "x.vcf"
    p.write_text(VCF)
    hm = haplotype_matrix.HaplotypeMatrix.from_vcf(str(p))
    assert hm.num_haplotypes == 6 and hm.num_variants == 5
    # first alleles of all samples, then second alleles (haplotype_matrix.py:326-329)
    np.testing.assert_array_equal(hm.haplotypes[:, 0], [0, 1, 0, 1, 1, 0])
    assert hm.haplotypes[0, 2] == -1
    f = hm.apply_biallelic_filter()
    keep = O.biallelic_keep(hm.haplotypes)
    np.testing.assert_array_equal(np.asarray(f.positions), hm.positions[keep])
    assert list(np.asarray(f.positions)) == [10, 40, 90]
    pf = tmp_path / "pops.txt"
    pf.write_text("sample\tpop\ns0\tA\ns1\tB\ns2\tA\n")
    hm.load_pop_file(str(pf))
    assert hm.sample_sets == {"A": [0, 3, 2, 5], "B": [1, 4]}
    gm = genotype_matrix.GenotypeMatrix.from_haplotype_matrix(f)
    np.testing.assert_array_equal(gm.genotypes[:, 0], [1, 1, 1])  # rows (0,1), (2,3), (4,5)


def test_genotype_filter_matches_oracle():
    rng = np.random.default_rng(1)
    g = rng.integers(-1, 3, size=(30, 200)).astype(np.int8)
    g[:, :20] = 0
    gm = genotype_matrix.GenotypeMatrix(g, np.arange(200))
    np.testing.assert_array_equal(gm.biallelic_keep(), O.geno_biallelic_keep(g))
    np.testing.assert_array_equal(gm.biallelic_keep(rows=range(10)), O.geno_biallelic_keep(g, range(10)))


def test_names_specs_match_reference(golden_dir):
    with open(os.path.join(golden_dir, "ref_names.json")) as f:
        ref = json.load(f)
    for P in (1, 2, 3, 4):
        assert ld_pipeline.ld_names(P) == ref[str(P)]["ld"]
        assert ld_pipeline.het_names(P) == ref[str(P)]["het"]
        mine = [[n, [[w, k, list(q)] for (w, k, q) in calls]] for n, calls in ld_pipeline.generate_stat_specs(P)]
        assert mine == ref[str(P)]["specs"]


def test_chunk_size_model():
    assert ld_pipeline.estimate_ld_chunk_size(100, available_memory_bytes=10 ** 9) == 10 ** 9 // ((4 * 100 * 2 + 300) * 3)
    assert ld_pipeline.estimate_ld_chunk_size(100, available_memory_bytes=10) == 100_000
    assert ld_pipeline.estimate_ld_chunk_size(1, available_memory_bytes=10 ** 13) == 10_000_000


def test_genetic_map_helpers(tmp_path):
    m = tmp_path / "map.txt"
    m.write_text("pos\tMap(cM)\n0\t0.0\n1000000\t1.0\n2000000\t3.0\n")
    pos = np.array([0, 500_000, 1_000_000, 1_500_000, 2_000_000])
    gen = moments_ld._interpolate_genetic_distances(pos, str(m))
    np.testing.assert_allclose(gen, [0.0, 0.005, 0.01, 0.02, 0.03])
    # slowest rate 1e-8 / bp: 1e-3 M -> 1e5 bp x 1.1
    assert abs(moments_ld._max_bp_for_r_dist(pos, gen, 1e-3) - 110_000.0) < 1e-6
    assert moments_ld._max_bp_for_r_dist(pos, gen, 10.0) == 2_000_000.0


def test_tc_blocks_fit_matches_the_kernel_rule():
    """Host check of the tensor-core row blocks' bootstrap-block span (64 / 128 SNPs from
    each window start may cover at most 2 / 4 blocks from their first SNP's block)."""
    from pg_gpu_b200.parse import tc_blocks_fit
    n = 300
    big = np.arange(n) // 100                      # 100-SNP blocks: a 64-SNP row block spans <= 2
    assert tc_blocks_fit(big, None, n) and tc_blocks_fit(big, None, n, genotypes=True)
    small = np.arange(n) // 30                     # 30-SNP blocks: 64 SNPs span 3
    assert not tc_blocks_fit(small, None, n)
    assert tc_blocks_fit(np.arange(n) // 40, None, n, genotypes=True)       # 128 SNPs span <= 4
    assert not tc_blocks_fit(np.arange(n) // 30, None, n, genotypes=True)   # ... but 5 here
    # row blocks restart at each window: windows of 60 SNPs keep 30-SNP blocks within two
    assert tc_blocks_fit(small, [0, 60, 120, 180, 240, 300], n)
    down = big.copy()
    down[5] = -1                                   # a block index below the row block's first
    assert not tc_blocks_fit(down, None, n)


def test_genotype_horner_forms_are_exact_in_fp64():
    """The generated Horner forms of the three single-population genotype polynomials give
    bit-identical FP64 results to pg_gpu's expanded forms on integer cell counts (every
    intermediate is an integer below 2^53 for counts up to 10^4)."""
    from pg_gpu_b200.csrc import gen_estimators as G

    class X:
        pass

    rng = np.random.default_rng(5)
    x = X()
    for m in range(1, 10):
        setattr(x, f"g{m}", rng.integers(0, 10_000, size=20_000).astype(np.float64))
    for poly in G._HORNER_POLYS.values():
        want = eval(poly, {}, {"x": x})
        got = eval(G.horner_form(poly), {}, {"x": x})
        np.testing.assert_array_equal(got, want)


def test_pack_codes_round_trip():
    """Two-bit packing of the ingest layout (LDK_X_PACKED2): code + 1 in bits 2 (v % 4) of
    byte v / 4; unpacking restores every code, at every n_var modulo 4."""
    from pg_gpu_b200 import parse
    rng = np.random.default_rng(7)
    for n_var in (1, 2, 3, 4, 5, 130):
        x = rng.integers(-1, 3, size=(9, n_var)).astype(np.int8)
        p = parse.pack_codes(x)
        assert p.dtype == np.uint8 and p.shape == (9, (n_var + 3) // 4)
        np.testing.assert_array_equal(parse.unpack_codes(p, n_var), x)
        v = n_var - 1
        np.testing.assert_array_equal((p[:, v // 4] >> (2 * (v % 4))) & 3, x[:, v] + 1)


def test_exact_int_to_double_identity():
    """The tensor-core epilogue converts counts with the 2^52 "magic number" method
    (ldk_common.cuh: i2d_exact): the bit pattern 0x43300000:(x ^ 2^31) is the double
    2^52 + 2^31 + x, and one subtraction returns x exactly.  Checked in NumPy's IEEE float64
    over the int32 range ends and random values."""
    rng = np.random.default_rng(3)
    x = np.concatenate([np.array([0, 1, -1, 2**31 - 1, -2**31], np.int64),
                        rng.integers(-2**31, 2**31, 200_000)]).astype(np.int32)
    bits = (np.uint64(0x43300000) << np.uint64(32)) | (x.view(np.uint32) ^ np.uint32(0x80000000)).astype(np.uint64)
    np.testing.assert_array_equal(bits.view(np.float64) - 4503601774854144.0, x.astype(np.float64))


def _header_constant(name):
    import re
    path = os.path.join(os.path.dirname(__file__), "..", "pg_gpu_b200", "csrc", "ldk_internal.h")
    with open(path) as f:
        return int(re.search(r"constexpr int %s = (\d+);" % name, f.read()).group(1))


def test_work_item_split_fits_its_capacity():
    """The tensor-core parse cuts each row block's partner tiles into runs of at most
    c = max(min_tiles, ceil(total / kItemTarget)) tiles, min_tiles >= kMinItemTiles set by
    the shape's staged sums; the workspace holds n_row_blocks + kItemTarget items.  The
    bound holds for any tile counts (sum of ceil(t / c) <= total / c + row blocks with
    tiles), checked here on skewed random shapes, and the runs of one row block cover its
    tiles exactly once."""
    target, cmin0 = _header_constant("kItemTarget"), _header_constant("kMinItemTiles")
    rng = np.random.default_rng(5)
    for trial in range(200):
        cmin = cmin0 if trial % 2 else int(rng.integers(cmin0, 40))
        n_rb = int(rng.integers(1, 20000))
        tiles = rng.integers(0, int(rng.choice([3, 40, 400, 5000])), size=n_rb)
        tiles[rng.random(n_rb) < 0.1] = 0  # row blocks without partners get no item
        total = int(tiles.sum())
        c = max(cmin, -(-total // target))
        parts = -(-tiles // c)
        assert parts.sum() <= n_rb + target
        for t in tiles[:50]:
            t = int(t)
            runs = [(q * c, t if q == -(-t // c) - 1 else (q + 1) * c) for q in range(-(-t // c))]
            covered = [x for a, b in runs for x in range(a, min(b, t))]
            assert covered == list(range(t))
