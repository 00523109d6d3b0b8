"""The sweep workload's problem draw (no GPU)."""
import sweep


def test_sweep_problem_draw_is_seeded_and_in_range():
    a = sweep.draw_problems(8, 1)
    b = sweep.draw_problems(8, 1)
    assert [(p.nx, p.ny, p.nz, p.rows, p.Ks_l) for p in a] == [(p.nx, p.ny, p.nz, p.rows, p.Ks_l) for p in b]
    for p in a:
        assert p.nx in sweep.SIZES_X and p.ny in sweep.SIZES_YZ and p.nz in sweep.SIZES_YZ
        assert 8 <= p.rows <= 40 and p.rows == p.cols and p.pinned == 1
        assert 0.55 <= p.tau <= 0.9 and 1e-3 <= p.Ks_l <= 1e-1 and 1e-4 <= p.Kb_l <= 1e-2
        assert 0.005 <= p.u_l <= 0.03
        assert p.y0 >= 2 and p.y0 + p.height <= p.ny - 3
