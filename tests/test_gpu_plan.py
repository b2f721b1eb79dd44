"""Database-search plans (parasail_b200_db_plan_*): the search recorded
once as a CUDA graph and replayed gives the records of
parasail_b200_batch_db_device, run after run, also after the target codes
change in place, and plans refuse the jobs the graph does not hold."""
import random

import numpy as np
import pytest

from conftest import AA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")
torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_plan_replays_equal_batch_db_device():
    rng = random.Random(31)
    b62 = pb.matrix_lookup("blosum62")
    mapper = np.ctypeslib.as_array(b62.contents.mapper, shape=(256,)).astype(np.uint8)
    queries = [rand_seq(rng, L, AA) for L in (40, 300, 1000)]
    targets = [mutate(rng, queries[k % 3], AA, 0.3, 0.03) if k % 5 == 0 else rand_seq(rng, rng.randint(10, 700), AA)
               for k in range(900)]
    buf, offs, lens = pb.pack(targets)
    # a second database of the same lengths, for the in-place update
    buf2 = np.frombuffer("".join(rand_seq(rng, int(l), AA) for l in lens).encode(), np.uint8).copy()
    profs = [pb.ProfileHandle("parasail_profile_create_sat", q, b62) for q in queries]
    parr = pb.ctypes.cast(pb.profile_array(profs), pb.ctypes.c_void_p)
    d_codes = torch.from_numpy(mapper[buf]).cuda()
    d_offs, d_lens = torch.from_numpy(offs).cuda(), torch.from_numpy(lens).cuda()
    n, nq = len(lens), len(queries)
    for name in ("sw_striped_profile_sat", "sw_scan_profile_16"):
        d_plan_rec = torch.zeros((nq, n, 8), dtype=torch.int32, device="cuda")
        d_ref_rec = torch.zeros((nq, n, 8), dtype=torch.int32, device="cuda")
        plan = pb.lib.parasail_b200_db_plan_create(name.encode(), parr, nq, d_codes.data_ptr(), d_offs.data_ptr(),
                                                   d_lens.data_ptr(), n, 11, 1, d_plan_rec.data_ptr())
        assert plan
        for codes in (buf, buf2, buf):
            d_codes.copy_(torch.from_numpy(mapper[codes]))
            for _ in range(2):
                d_plan_rec.zero_()
                assert pb.lib.parasail_b200_db_plan_run(plan) == 0
                assert pb.lib.parasail_b200_batch_db_device(name.encode(), parr, nq, d_codes.data_ptr(),
                                                            d_offs.data_ptr(), d_lens.data_ptr(), n, 11, 1,
                                                            d_ref_rec.data_ptr()) == 0
                torch.cuda.synchronize()
                assert torch.equal(d_plan_rec, d_ref_rec), name
            # the same search from host memory: characters in, records out
            h_rec = np.zeros((nq, n, 8), np.int32)
            assert pb.lib.parasail_b200_db_plan_run_host(plan, codes.ctypes.data, len(codes), h_rec.ctypes.data) == 0
            assert (h_rec == d_ref_rec.cpu().numpy()).all(), name
            assert (d_codes.cpu().numpy() == mapper[codes]).all()
        pb.lib.parasail_b200_db_plan_free(plan)
    # jobs a plan does not hold
    for name, op, gp in (("sw_stats_striped_profile_16", 11, 1), ("nw_scan_profile_16", 11, 1),
                         ("sw_striped_profile_16", 1, 1)):
        d_rec = torch.zeros((nq, n, 8), dtype=torch.int32, device="cuda")
        assert not pb.lib.parasail_b200_db_plan_create(name.encode(), parr, nq, d_codes.data_ptr(),
                                                       d_offs.data_ptr(), d_lens.data_ptr(), n, op, gp,
                                                       d_rec.data_ptr())
    for p in profs:
        p.close()
