"""CPU oracle for Harmony's IVF query path — TEST INFRASTRUCTURE ONLY.

Two libraries live here, both used only as checkers (by ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline / reference arm):

* ``oracle.ref``  — the reference's own C++ (``harmony::Index`` and friends)
  compiled unmodified from the reference sources into ``oracle/_ref``.
* ``oracle.port`` — this project's sequential C++ restatement of the same
  algorithm (``oracle/hy_oracle.cpp``), built into ``oracle/_build``.
* ``oracle.gpu_bruteforce`` — float64 brute force on the GPU (torch), the
  recall and distance-error oracle of the full-size measurement.
* ``oracle.mlp``  — numpy restatement of the learned probe predictor
  (features, stop labels, network forward/backward) for checking its kernels.

The product library (``harmonyclient_b200``) never imports this package.
"""
