"""The three forms beside the plain drop-in: ``precision`` (FP32 fluxes with
FP64 state, RK and pressure recovery), ``ensemble`` (batches of independent
boxes in one persistent launch per RK stage) and ``closure`` (a learned
per-element RHS correction for under-resolved runs)."""
