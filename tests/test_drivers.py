"""The run drivers a user starts from the command line: `python -m dnds_b200.explicit` (SSP-RK3 runs of
the vortex and the Riemann problem, the role of the reference's explicit solver loop) and
`python -m dnds_b200.steady` (the implicit steady run, here with the partitioned sweep).  Small cases:
they run, report no flagged flux and print their figures."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["vortex", "riemann"])
def test_explicit_driver_runs(case, capsys):
    from dnds_b200 import explicit

    assert explicit.main(["--case", case, "--grid", "16", "--steps", "2", "--warmup", "1",
                          "--limiter-all", "1" if case == "riemann" else "0"]) == 0
    out = capsys.readouterr().out
    assert "ms per step" in out and ("limiter, every cell" in out) == (case == "riemann")


def test_steady_driver_partitioned_sweep_runs(capsys):
    from dnds_b200 import steady

    assert steady.main(["--case", "euler", "--iters", "3", "--every", "1", "--parts", "4"]) == 0
    out = capsys.readouterr().out
    assert "done: 3 iterations" in out
