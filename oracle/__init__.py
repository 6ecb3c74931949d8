"""Test infrastructure only: CPU checkers for the GPU evaluator.

* ``oracle.cpu`` -- ctypes front end of ``liboracle.so``, the C restatement of
  the reference's per-point algorithms (agb_oracle.c);
* ``oracle.refpy`` -- the reference's own Python and kernels run on the CPU
  (needs the reference sources; used to produce golden vectors).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package.
"""
