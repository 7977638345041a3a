"""B200 (sm_100a) backend of gpumetropolis's sampler hot path.

``gpum_model`` compiles a formula to the reference's stack-machine bytecode;
``gpu_metropolis`` runs the batched sampler through the C-ABI library
(``libgpum_b200.so``, loaded on first use).
"""
from .api import (GpumBayesFactor, GpumEvidence, GpumFit, GpumInputError, gpu_metropolis,
                  gpum_bayes_factor, gpum_evidence)
from .dsl import gpum_model

__all__ = ["gpum_model", "gpu_metropolis", "gpum_evidence", "gpum_bayes_factor", "GpumFit",
           "GpumEvidence", "GpumBayesFactor", "GpumInputError"]
