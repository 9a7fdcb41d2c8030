"""Oracles of the reference's shallow-water step. TEST INFRASTRUCTURE ONLY.

``fp64_step`` restates the reference's float64 CPU step
(``tests/unit/_cpu_step.py``); ``fp32_resident.c`` with ``resident_oracle``
restates its float32 GPU-resident kernels. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline arm use them.
"""
