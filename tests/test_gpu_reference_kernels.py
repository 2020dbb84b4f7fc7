"""The reference's own CUDA path built for sm_100a (oracle/_ref/plfbs_ref_gpu:
Solver_gpu.cu and the kernels it launches, unmodified, as one translation
unit) run as the reference program on the golden cases, against the fixtures
that the host-serial run of the same kernels produced: the second FP64 parity
target of the library, agreeing to rounding (device FMA contraction and the
order of the reference's CAS atomics). The kernels' accesses on these inputs
were checked on the host under AddressSanitizer (make -C oracle/ref asan).
Skipped when the binary was not built (it needs the reference sources)."""

import os

import pytest

import golden_cases
import refrun
from conftest import REPO, load_golden, rel_l2

pytestmark = pytest.mark.gpu

BIN_GPU = os.path.join(REPO, "oracle", "_ref", "plfbs_ref_gpu")


@pytest.mark.parametrize("name", golden_cases.NAMES)
def test_reference_cuda_path_matches_the_fixtures(tmp_path, name):
    if not os.path.exists(BIN_GPU):
        pytest.skip("oracle/_ref/plfbs_ref_gpu not built (needs the reference sources)")
    d = golden_cases.build(name)
    g = load_golden(name)
    dumps = refrun.run_reference(str(tmp_path), d["pm"], d["case"], nodes=d["nodes"],
                                 init_state=d["state0"], binary=BIN_GPU, timeout=300)
    st = dumps["ref_gpu_final_state"]
    assert st.shape == g["final_state"].shape
    # after a converged exit the reference re-applies its host boundary update
    # to soln's ghosts (Solver_gpu.cu:872-881); the fixture holds the device
    # state, so ghosts are compared only for runs that ended out of time
    converged = int(g["steps_done"][0]) < d["case"].steps
    n = d["ma"].n_cells if converged else st.shape[0]
    for k in range(4):
        assert rel_l2(st[:n, k], g["final_state"][:n, k]) < 1e-10, k
