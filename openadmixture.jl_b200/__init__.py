"""B200-native engine for OpenADMIXTURE.jl's likelihood / gradient / Hessian sweeps, block SQP
updates and ZAL quasi-Newton extrapolation.

The engine is ``lib/libadmix.so`` (C ABI in ``include/admix.h``); this package is the host
side that mirrors the reference's Julia API over it.  Import it as ``openadmixture_b200``
(the repository root holds an import shim of that name).
"""
from . import _native
from ._native import AdmixError, IterInfo, ADMIX_FLAG_MIXED, ADMIX_FLAG_MU_GERSHGORIN, ADMIX_FLAG_MEAN_IMPUTE
from .admixture import (AdmixData, CuAdmixData, X, X_NEXT, X_NEXT2, X_TMP, _cu_admixture_base,
                        admixture_qn, em_p, em_q, init_em, loglikelihood, run_admixture, skfr, update_p,
                        update_q)
from .bed import BedFormatError, DeviceGenotypes, Genotypes, read_bed, write_bed
from .synth import COHORTS, CohortSpec, genotypes, genotypes_device, init_x, make_cohort, truth
from . import warmstart
from .batch import AdmixBatch, BatchMember, k_sweep, run_restarts

__all__ = [
    "AdmixData", "CuAdmixData", "AdmixError", "IterInfo", "Genotypes", "DeviceGenotypes", "BedFormatError",
    "X", "X_NEXT", "X_NEXT2", "X_TMP", "ADMIX_FLAG_MIXED", "ADMIX_FLAG_MU_GERSHGORIN", "ADMIX_FLAG_MEAN_IMPUTE",
    "_cu_admixture_base", "admixture_qn", "em_p", "em_q", "init_em", "loglikelihood",
    "run_admixture", "skfr", "update_p", "update_q", "read_bed", "write_bed",
    "COHORTS", "CohortSpec", "genotypes", "genotypes_device", "init_x", "make_cohort", "truth",
    "warmstart", "AdmixBatch", "BatchMember", "k_sweep", "run_restarts",
]
