"""The largest pictures a session takes: 4,096 MBs, the most a work item's
12-bit MB index addresses.  A square 1024x1024 picture and a 4096x256 strip
(256 MBs per row) encode bit for bit as the oracle does -- records, levels
and reconstructions, an intra picture and two inter ones, in a step beside a
QCIF session -- and a picture of 4,160 MBs is refused at open."""
import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import synth
from h261enc_cuda_b200._lib import H261Error
from h261enc_cuda_b200.engine import Engine

pytestmark = pytest.mark.gpu
N = 3


@pytest.mark.parametrize("w,h", [(1024, 1024), (4096, 256)])
def test_largest_pictures_match_oracle(gpu, w, h):
    big = synth.clip(1, w, h, 71 + w, N)
    small = synth.clip(2, 176, 144, 72, N)
    want_big = O.encode_sequence(big, w, h, 9)
    want_small = O.encode_sequence(small, 176, 144, 14)
    with Engine(max_sessions=4) as e:
        sb = e.open(w, h, 9)
        ss = e.open(176, 144, 14)
        for i in range(N):
            e.submit_frames([sb, ss], [big[i], small[i]])
            e.step()
            e.sync()
            for sid, want, ww in ((sb, want_big, w), (ss, want_small, 176)):
                r = e.result(sid)
                got = r.to_abi(ww)
                for f in ("type", "flags", "quant", "cbp", "mv", "tcoeff"):
                    assert np.array_equal(got[f], want["mbs"][i][f]), f"{ww}: picture {i}: field {f}"
                assert np.array_equal(np.concatenate(e.recon(sid)), want["recon"][i]), \
                    f"{ww}: picture {i}: reconstruction"


def test_picture_over_4096_mbs_is_refused(gpu):
    with Engine(max_sessions=4) as e:
        with pytest.raises(H261Error):
            e.open(1040, 1024, 8)      # 65 x 64 = 4,160 MBs
        sid = e.open(1024, 1024, 8)    # 4,096: taken
        assert sid >= 0
