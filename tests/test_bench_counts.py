"""The bench's per-launch byte counts and launch counts (host logic, no GPU): the ROMS form's
rhs3d and column solve move what their kernels read and write, and a ROMS-form step launches
7 kernels plus four per barotropic substep (the last substep: the predictor's averages only)."""
import os
import sys
import types

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def _grid(L, M, N):
    return types.SimpleNamespace(L=L, M=M, N=N, s2=(L + 1) * (M + 1))


def test_algorithmic_bytes_of_the_roms_form():
    import bench
    g = _grid(101, 51, 20)
    s2, N = g.s2, g.N
    ref = bench.algorithmic_bytes(g, 4)
    roms = bench.algorithmic_bytes(g, 4, "roms")
    # the ROMS rhs3d reads no W (its vertical advection is in the column solve)
    assert roms["k_rhs3d"] == ref["k_rhs3d"] - 4 * N * s2
    # the ROMS column solve reads three right-hand-side slots per component and W
    assert roms["k_step3d_uv"] == 4 * (14 * N + 4) * s2 + 16 * s2
    assert roms["k_maxflux_omega"] == ref["k_maxflux_omega"]
    assert roms["k_set_depth"] == ref["k_set_depth"]


def test_launches_per_step_of_the_roms_form():
    import bench
    m = types.SimpleNamespace(semantics="roms", nfast=42)
    assert bench.launches_per_step(m, "none") == 7 + 4 * 42 + 1
    assert bench.launches_per_step(m, "mlp") == 7 + 4 * 42 + 1 + 3
