"""B200 (sm_100a) prover core for Neo lattice folding: Ajtai commitment and
batched sum-check, exposed through the C ABI in include/neo_gpu.h."""
from .params import GOLDILOCKS, NeoParams, D, Q  # noqa: F401
