"""B200-native MLS-MPM substep of litter-physics (CUDA for sm_100a behind a C ABI).

Modules:
  _abi      ctypes mirrors of the POD structs in include/lp_mpm.h
  _lib      loader of the device library and status checking
  sim       Simulation / Batch: the reference's Simulation API over the device library
  research  research wire request -> fixture spec (research.rs:171-305)
  configs   the benchmark workloads (slump, dam break, large slump, batched sweep, pellet bed)
  _core     drop-in `protocol_version` / `run_json` of the reference's `_core` module
  warmstart Newton-pair collection and device training of the warm-start network
  sweep, verification  parameter sweeps and refinement studies on the batched launch
"""

from ._abi import FixtureSpec, Ledger, Material  # noqa: F401

__all__ = ["FixtureSpec", "Ledger", "Material"]
