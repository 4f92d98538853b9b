"""The file-to-file application (h261enc_cuda_b200/app.py): YUV reading and
writing as the reference's main does it, and, on the GPU, a whole file
encoded to the reference encoder's bitstream, reconstruction and PSNR."""
import os

import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import app, synth


def test_yuv_roundtrip_and_partial_tail(tmp_path):
    fr = synth.clip(0, 176, 144, 3, 4)
    p = str(tmp_path / "a.yuv")
    app.write_yuv(p, fr)
    with open(p, "ab") as f:
        f.write(b"\x01" * 1000)            # a partial picture at the end is not read
    back = app.read_yuv(p, 176, 144)
    assert back.shape == fr.shape and np.array_equal(back, fr)
    assert np.array_equal(np.stack(list(app.iter_yuv(p, 176, 144))), fr)
    assert app.read_yuv(p, 176, 144, max_frames=2).shape[0] == 2


def test_statistics_line_format():
    st = app.PictureStats(3, 12, 39600, 4096, (34.5, 40.25, 41.0), 1.2345)
    assert st.line() == ("frame 0003, quant=12, cost=39600, size=4096, ypsnr=34.500000, cbpsnr=40.250000, "
                         "crpsnr=41.000000, time=1.234ms")


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,quant,bitrate,intra", [(352, 288, 0, 512000, 0), (176, 144, 9, 0, 5)])
def test_encode_file_matches_reference_frame_loop(gpu, tmp_path, w, h, quant, bitrate, intra):
    fr = synth.clip(1 if w == 352 else 0, w, h, 11, 9)
    src, bits, rec = (str(tmp_path / n) for n in ("in.yuv", "out.h261", "rec.yuv"))
    app.write_yuv(src, fr)
    lines = []
    stats = app.encode_file(src, bits, rec, w, h, quant=quant, bitrate=bitrate, intra_period=intra,
                            log=lines.append)
    want_bits, want_nb, want_q, want_rec = O.encode_stream(fr, w, h, quant=quant, bitrate=bitrate or 384000,
                                                           intra_period=intra)
    assert open(bits, "rb").read() == want_bits
    got_rec = app.read_yuv(rec, w, h)
    assert np.array_equal(got_rec, want_rec)
    for i, st in enumerate(stats):
        assert st.quant == want_q[i] and st.size == want_nb[i]
        assert st.psnr == O.psnr(fr[i], want_rec[i], w, h)[1], f"picture {i}: PSNR"
    assert len(lines) == len(stats) + 2 and lines[-2].startswith("PSNR Mean:")
    os.remove(src)
