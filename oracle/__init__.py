"""CPU oracle for the particle-filter hot path -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg (and its ``--impl reference`` arm) may import, call, link or execute
anything in this directory.  The shipped package never does: its compute path
is the CUDA library and fails loudly when that library is missing.

Contents:
  jaxrng.py     JAX's Threefry streams restated (pins fixtures to the reference)
  models_np.py  float32 NumPy models (LG / SV / Ricker)
  refpath.py    float32 NumPy restatement of pfilter / mop / simulate
  kalman.py     FP64 Kalman filter (exact LG log-likelihood)
  ppf_oracle.c  C restatement with the CUDA path's exact arithmetic
                (fixed-point CDF, Philox4x32-10) for bit-exact comparisons
"""
