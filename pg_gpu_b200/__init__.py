"""pg_gpu_b200: B200-native (sm_100a) two-locus LD parse with pg_gpu's call surface.

The compute lives in ``libldk.so`` (CUDA C++, C ABI in ``include/ldk.h``); these modules
are the host side: ``ld_pipeline`` / ``ld_statistics`` / ``moments_ld`` /
``haplotype_matrix`` / ``genotype_matrix`` mirror pg_gpu's LD interface, ``parse`` is the
binned parse, ``synth`` the seeded synthetic workloads.
"""
__version__ = "0.1.0"
