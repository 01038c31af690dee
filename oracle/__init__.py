"""CPU oracle for the SawSim frequency-sweep hot path — TEST INFRASTRUCTURE ONLY.

A NumPy/SciPy restatement of the reference's algorithm (Duane245/sawsim 2.1.0),
each function citing the reference file:line it follows.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may
import it, and only as the checker or the timed CPU baseline.  The product
package ``sawsim_b200`` never imports it; its sweep runs on the GPU only.

Pinned against the reference in two ways (see tests/test_oracle_pins.py):

* the published golden curve ``tests/data/sp_double_layer.npz`` of the reference
  (``sawsim_magnitude`` at the 5 test frequencies), rebuilt here without Gmsh;
* matrices, charges and admittances produced by importing the reference itself
  in the build container, committed as fixtures under ``tests/golden/`` with the
  script that generated them (``tests/golden/make_golden.py``).
"""
