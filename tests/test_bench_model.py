"""The bench's accounting: the kernel-launch count and the compulsory-bytes
model (``roofline.achieved``) reproduce the figures of a recorded bench line
from its device counters (128x128x32 film, 499,999 interior nodes, 20 steps,
mixed precision, GMRES with the degree-10 polynomial preconditioner)."""

import bench

N_INT = 499_999
COUNTERS = {"steps": 20, "rejections": 0, "newton_iters": 41, "krylov_iters": 82, "krylov_sq": 204,
            "rhs_evals": 81, "jvp_evals": 902}


def test_launch_count_of_the_recorded_line():
    # 7 per step, 4 per Newton iteration, 4 + 10 per Arnoldi step (one more than the iterations per solve)
    assert bench.graph_launches(COUNTERS, "analytic", 10) == 7 * 20 + 4 * 41 + 14 * (82 + 41) == 2026
    assert bench.graph_launches(COUNTERS, "fd") == 7 * 20 + 4 * 41 + 5 * 82


def test_compulsory_bytes_of_the_recorded_line():
    alg = bench.algorithmic_bytes(N_INT, "mixed", COUNTERS, 10)
    assert alg == 52_511_394_977.0
    # each preconditioner step reads the vector it preconditions: 1 FP32 vector per Horner step
    assert alg - bench.algorithmic_bytes(N_INT, "mixed", COUNTERS, 0) == 10 * 82 * 20.0 * N_INT
    # FP64 Krylov vectors double the Krylov terms only
    fp64 = bench.algorithmic_bytes(N_INT, "fp64", COUNTERS, 10)
    sk = 20.0 * N_INT
    assert fp64 - alg == 902 * 3 * sk + (204 + 7 * 82) * sk + 10 * 82 * sk

