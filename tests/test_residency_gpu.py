"""Residency of the step kernels (sh_residency): the register budgets and the
shared-memory sizing of the 256^3 FP32 step hold three CTAs per SM in both
passes, and the reported waves follow from the grid sizes."""
import pytest

import smectic3d_b200 as S

pytestmark = pytest.mark.gpu


def test_residency_256_fp32_three_ctas_per_sm():
    torch = pytest.importorskip("torch")
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    with S.Solver(S.Params(n=256, boundary="neumann", precision="fp32")) as s:
        r = s.residency()
    assert r["sms"] == sms
    assert r["plane_ctas_per_sm"] == 3 and r["pencil_ctas_per_sm"] == 3
    assert r["plane_cluster"] == 8 and r["plane_ctas"] == 256 * 8
    assert r["pencil_ctas"] == 256 * 128 // 16
    # whole clusters only: never more CTAs than the SMs hold
    assert 1 <= r["plane_clusters_resident"] * 8 <= 3 * sms
    assert r["plane_waves"] == pytest.approx(2048 / (8 * r["plane_clusters_resident"]))
    assert r["pencil_waves"] == pytest.approx(2048 / (3 * sms))


def test_residency_unclustered_counts_every_slot():
    with S.Solver(S.Params(n=32, boundary="periodic", precision="fp64", batch=4)) as s:
        r = s.residency()
    assert r["plane_cluster"] == 1 and r["plane_ctas"] == 32 * 4
    assert r["plane_clusters_resident"] == r["plane_ctas_per_sm"] * r["sms"]
    assert r["pencil_ctas_per_sm"] >= 1


def test_residency_256_fp64_neumann_reads_twiddles_in_place():
    """FP64 Neumann 256^3 (clusters of 16): with its 7.9 KB of twiddles read from
    the device table instead of shared memory, three CTAs fit an SM; the periodic
    plane pass, register-bound at two, keeps them in shared memory."""
    with S.Solver(S.Params(n=256, boundary="neumann", precision="fp64")) as s:
        r = s.residency()
    assert r["plane_cluster"] == 16 and r["plane_ctas_per_sm"] == 3
    with S.Solver(S.Params(n=256, boundary="periodic", precision="fp64")) as s:
        r = s.residency()
    assert r["plane_cluster"] == 16 and r["plane_ctas_per_sm"] == 2
