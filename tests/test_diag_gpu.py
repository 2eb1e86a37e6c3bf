"""GPU tests of the random-access microbenchmark (pg_diag_random_access).

It measures the rates the filters' kernels are judged against, so it must
do the accesses it reports: every mode runs and returns the count it
launched, the atomic-add mode's adds all land (the buffer's words sum to the
count), the modes that write change the buffer, and bad arguments are
refused before anything runs."""
import pytest

pytestmark = pytest.mark.gpu


def _modes(pg):
    return [pg.PG_DIAG_READ32, pg.PG_DIAG_READ64, pg.PG_DIAG_READ32_CAS, pg.PG_DIAG_RED32,
            pg.PG_DIAG_READ32_CAS_NEXT]


def test_every_mode_runs_and_reports_its_accesses(pg):
    import torch
    for mode in _modes(pg):
        buf = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
        done = pg.diag_random_access(buf, mode, 100_000, seed=mode + 1, blocks_per_sm=2)
        torch.cuda.synchronize()
        assert done >= 100_000
        words = buf.view(torch.int32)
        if mode == pg.PG_DIAG_RED32:
            # one atomic add of 1 per access, none lost
            assert int(words.sum().item()) == done
        elif mode in (pg.PG_DIAG_READ32_CAS, pg.PG_DIAG_READ32_CAS_NEXT):
            # each CAS from the value read to one more: at most one per access
            assert 0 < int(words.sum().item()) <= done
        else:
            assert int(words.abs().sum().item()) == 0  # reads leave the buffer alone


def test_bad_arguments_are_refused(pg):
    import torch
    buf = torch.zeros(1 << 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(pg.PoggersError):
        pg.diag_random_access(buf, 5, 1000)  # no such mode
    with pytest.raises(pg.PoggersError):
        pg.diag_random_access(buf[1:1025], pg.PG_DIAG_READ32, 1000)  # not 64-byte aligned
    with pytest.raises(pg.PoggersError):
        pg.diag_random_access(buf[:32], pg.PG_DIAG_READ32, 1000)  # under 64 bytes
    with pytest.raises(pg.PoggersError):
        pg.diag_random_access(buf, pg.PG_DIAG_READ32, 1000, blocks_per_sm=9)  # more than an SM holds
