"""Drop-in for ``pg_gpu.ld_statistics_genotype``'s all-pairs entry point
(``sigma_d2_geno``, ``pg_gpu/ld_statistics_genotype.py:1518-1598``) on libldk's genotype
all-pairs kernel."""
from __future__ import annotations

from .ld_matrix import sigma_d2_geno  # noqa: F401
