"""parasail_b200_batch_profile_device_noalloc, called through the C ABI,
against parasail_b200_batch_profile_device on the same device-resident
inputs: two different batches in a row (and the first again), so that a
call that read what the previous call left in the static scratch would
show; then the limits it must reject.

Collected last on purpose: it must pass both alone in a fresh process and
after every other test has used the device."""
import random

import numpy as np
import pytest

from conftest import AA, rand_seq, mutate

pb = pytest.importorskip("parasail_b200")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CASES = [("sw_striped_profile_16", "parasail_profile_create_16"),
         ("sw_scan_profile_sat", "parasail_profile_create_sat"),
         ("nw_scan_profile_sat", "parasail_profile_create_sat"),
         ("sg_qb_de_striped_profile_8", "parasail_profile_create_8"),
         ("sg_qx_stats_striped_profile_16", "parasail_profile_create_stats_16"),
         ("nw_stats_scan_profile_sat", "parasail_profile_create_stats_sat"),
         ("sw_stats_scan_profile_32", "parasail_profile_create_stats_32")]


def _device_targets(targets, matrix):
    buf, offs, lens = pb.pack(targets)
    mapper = np.ctypeslib.as_array(matrix.contents.mapper, shape=(256,)).astype(np.uint8)
    codes = mapper[buf]
    return (torch.from_numpy(codes).cuda(), torch.from_numpy(offs).cuda(), torch.from_numpy(lens).cuda())


def _call(entry, name, prof, dev, open_, gap):
    n = dev[2].numel()
    rec = torch.full((n, 8), -7, dtype=torch.int32, device="cuda")
    rc = entry(name.encode(), prof.ptr, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), n, open_, gap,
               rec.data_ptr())
    torch.cuda.synchronize()
    return rc, rec.cpu().numpy().view(pb.record_dtype()).reshape(n)


def _dicts(recs, name):
    return pb.records_to_dicts(recs, "stats" in name)


def test_noalloc_equals_device_entry_two_calls_in_a_row():
    rng = random.Random(31)
    b62 = pb.matrix_lookup("blosum62")
    q = rand_seq(rng, 190, AA)
    batch_a = [mutate(rng, q, AA, 0.3, 0.05) if k % 2 else rand_seq(rng, rng.randint(1, 600), AA)
               for k in range(500)]
    batch_b = [rand_seq(rng, rng.randint(1, 120), AA) for _ in range(77)] + [q, q[::-1]]
    dev_a, dev_b = _device_targets(batch_a, b62), _device_targets(batch_b, b62)
    for name, creator in CASES:
        prof = pb.ProfileHandle(creator, q, b62)
        rc, na1 = _call(pb.lib.parasail_b200_batch_profile_device_noalloc, name, prof, dev_a, 11, 1)
        assert rc == 0, name
        rc, nb = _call(pb.lib.parasail_b200_batch_profile_device_noalloc, name, prof, dev_b, 11, 1)
        assert rc == 0, name
        rc, na2 = _call(pb.lib.parasail_b200_batch_profile_device_noalloc, name, prof, dev_a, 11, 1)
        assert rc == 0, name
        rc, ea = _call(pb.lib.parasail_b200_batch_profile_device, name, prof, dev_a, 11, 1)
        assert rc == 0, name
        rc, eb = _call(pb.lib.parasail_b200_batch_profile_device, name, prof, dev_b, 11, 1)
        assert rc == 0, name
        assert _dicts(na1, name) == _dicts(ea, name), name
        assert _dicts(nb, name) == _dicts(eb, name), name
        assert _dicts(na2, name) == _dicts(ea, name), name
        prof.close()


def test_noalloc_rejects_what_does_not_fit():
    rng = random.Random(32)
    b62 = pb.matrix_lookup("blosum62")
    q = rand_seq(rng, 50, AA)
    prof = pb.ProfileHandle("parasail_profile_create_16", q, b62)
    cap = pb.lib.parasail_b200_noalloc_scratch_bytes()
    assert cap == 32 << 20
    fn = pb.lib.parasail_b200_batch_profile_device_noalloc
    # more target residues than the strip buffers hold: rejected after the
    # length scan, before any alignment kernel reads a target
    n, each = 1000, 5000
    codes = torch.zeros(n * each, dtype=torch.uint8, device="cuda")
    offs = torch.arange(n, dtype=torch.int64, device="cuda") * each
    lens = torch.full((n,), each, dtype=torch.int32, device="cuda")
    rec = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
    assert fn(b"sw_striped_profile_16", prof.ptr, codes.data_ptr(), offs.data_ptr(), lens.data_ptr(), n, 11, 1,
              rec.data_ptr()) == -1
    # within the limit the same arrays align
    assert fn(b"sw_striped_profile_16", prof.ptr, codes.data_ptr(), offs.data_ptr(), lens.data_ptr(), 100, 11, 1,
              rec.data_ptr()) == 0
    # more pairs than the per-pair regions hold: rejected on the host
    big = 200000
    lens2 = torch.ones(big, dtype=torch.int32, device="cuda")
    offs2 = torch.zeros(big, dtype=torch.int64, device="cuda")
    rec2 = torch.zeros((big, 8), dtype=torch.int32, device="cuda")
    assert fn(b"sw_striped_profile_16", prof.ptr, codes.data_ptr(), offs2.data_ptr(), lens2.data_ptr(), big, 11, 1,
              rec2.data_ptr()) == -1
    # the two-pass statistics pipeline is not run here
    sprof = pb.ProfileHandle("parasail_profile_create_stats_16", q, b62)
    assert fn(b"sw_stats_striped_profile_16", sprof.ptr, codes.data_ptr(), offs.data_ptr(), lens.data_ptr(), 10, 11,
              1, rec.data_ptr()) == -1
    torch.cuda.synchronize()
    sprof.close()
    prof.close()
