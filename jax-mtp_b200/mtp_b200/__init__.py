"""B200 (sm_100a) Moment Tensor Potential engine: Python front end.

Modules:
    engine       MTPEngine: the C ABI of libmtp_b200.so (host and device entry points),
                 pinned_empty (page-locked NumPy arrays)
    md           DeviceMD: device-resident velocity-Verlet MD under CUDA graphs
    train        MTPFunction (batched forward + hand-written adjoint), losses,
                 least-squares basis solve, L-BFGS
    mtp_file     .mtp potential reader/writer
    cfg_file     MLIP .cfg configuration reader/writer
    synth        lattices, periodic neighbour rows, ghosts and full lists,
                 synthetic training batches
    autotune     launch-shape autotuner with an on-disk cache
    lammps_data  LAMMPS data-file reader
    profile_case bounded evaluation / adjoint / pair-style-call cases for profilers

The shared library is loaded on first use (``mtp_b200._lib.lib()``); every
entry point fails with a clear error if it has not been built.
"""
