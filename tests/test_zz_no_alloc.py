"""sbp_mdl_device_static: the MDL of a device-resident blockmodel computed
with no allocation inside the call, for callers that cannot let a library
allocate device memory (a host-owned memory pool, a serving loop that
forbids allocation syncs).  Checked against sbp_mdl (the allocating entry
point) and the CPU oracle on the same partitions, twice in a row so that the
scratch left by one call cannot leak into the next.  Named to be collected
last."""
import numpy as np
import pytest

from tests.graphs import dcsbm

REL = 1e-9


def _device_blockmodel(sbp, g, part, B):
    import torch
    bm = sbp.build_blockmodel(g, part, B)
    dev = {k: torch.from_numpy(np.ascontiguousarray(bm[k]).view(np.int32)).cuda()
           for k in ("optr", "ocol", "ocnt", "d_out", "d_in")}
    return dev


@pytest.mark.gpu
@pytest.mark.parametrize("variant,N,B", [("LL", 1000, 11), ("HH", 4000, 64), ("LH", 4000, 4000)])
def test_mdl_device_static_matches_mdl(sbp, orc, variant, N, B):
    import torch
    g = dcsbm(variant, N, seed=7)
    rng = np.random.default_rng(3)
    parts = [rng.integers(0, B, g.N).astype(np.int32), np.asarray(g.true_partitions, np.int32)]
    parts[0][:B] = np.arange(B)
    for part in parts:
        Bp = int(part.max()) + 1
        S_ref, data_ref = sbp.mdl(g, part, Bp)
        S_orc, data_orc = orc.mdl(g, part, Bp)
        dev = _device_blockmodel(sbp, g, part, Bp)
        out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
        for _ in range(2):
            out.fill_(float("nan"))
            stream = torch.cuda.current_stream().cuda_stream
            sbp.mdl_device_static(g.N, g.E, Bp, dev["optr"].data_ptr(), dev["ocol"].data_ptr(),
                                  dev["ocnt"].data_ptr(), dev["d_out"].data_ptr(),
                                  dev["d_in"].data_ptr(), out[0:1].data_ptr(),
                                  out[1:2].data_ptr(), stream)
            torch.cuda.synchronize()
            S, data_S = out.cpu().tolist()
            assert abs(S - S_ref) <= REL * abs(S_ref), (S, S_ref)
            assert abs(data_S - data_ref) <= REL * abs(data_ref), (data_S, data_ref)
            assert abs(S - S_orc) <= REL * abs(S_orc), (S, S_orc)
            assert abs(data_S - data_orc) <= REL * abs(data_orc), (data_S, data_orc)


@pytest.mark.gpu
def test_mdl_device_static_rejects_too_many_blocks(sbp):
    import torch
    z = torch.zeros(4, dtype=torch.int32, device="cuda")
    d = torch.zeros(2, dtype=torch.float64, device="cuda")
    with pytest.raises(sbp.SbpError, match="static scratch"):
        sbp.mdl_device_static(10, 10, 65537, z.data_ptr(), z.data_ptr(), z.data_ptr(),
                              z.data_ptr(), z.data_ptr(), d[0:1].data_ptr(), d[1:2].data_ptr(), 0)
    with pytest.raises(sbp.SbpError, match="bad arguments"):
        sbp.mdl_device_static(10, 10, 4, z.data_ptr(), 0, z.data_ptr(), z.data_ptr(),
                              z.data_ptr(), d[0:1].data_ptr(), d[1:2].data_ptr(), 0)
