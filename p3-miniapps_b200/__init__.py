"""vlp4d on B200: the semi-Lagrangian hot path of yasahi-hpc/P3-miniapps' vlp4d.

The product is the CUDA library libvlp4d_b200.so (C ABI in
include/vlp4d_b200.h, C++ reference-facing layer in cpp/).  This package
exposes its ctypes binding (``vlp4d``) for tests and benchmarks.

The directory name contains a hyphen, so it is loaded by path:
``__graft_entry__.load_package()`` registers it as ``p3_miniapps_b200``.
"""
from . import vlp4d  # noqa: F401
from .vlp4d import (Adjoint, Context, Domain, Ensemble, EnsembleMember, build, energy_after_steps,  # noqa: F401
                    landau_domain, landau_ensemble_members, lib)
