"""The conformance decoder (oracle/h261_decoder.c): H.261 streams written
by the oracle's restatement of the reference encoder parse back into the
encoder's records and reconstruct to the encoder's own reconstructions, bit
for bit."""
import numpy as np
import pytest

import oracle as O
from h261enc_cuda_b200 import synth

CASES = [(0, 176, 144, 8, 0, 0), (1, 352, 288, 0, 384000, 5), (3, 176, 144, 1, 0, 3), (0, 176, 144, 31, 0, 2),
         (2, 352, 288, 2, 0, 4), (0, 176, 144, 0, 32000, 0)]


def coded_equal(enc, dec):
    """Records agree on everything the syntax carries: uncoded blocks of an
    inter MB are not transmitted, whatever levels the encoder kept there."""
    for f in ("type", "flags", "quant", "cbp", "mv", "mb_x", "mb_y"):
        if not np.array_equal(enc[f], dec[f]):
            return False
    cbp = enc["cbp"]
    for b in range(6):
        coded = (cbp & (32 >> b)) != 0
        if not np.array_equal(enc["tcoeff"][coded, b], dec["tcoeff"][coded, b]):
            return False
    return True


@pytest.mark.parametrize("preset,w,h,quant,bitrate,intra", CASES)
def test_decoder_reconstructs_oracle_stream(preset, w, h, quant, bitrate, intra):
    fr = synth.clip(preset, w, h, 7, 6)
    bits, nbytes, quants, recon = O.encode_stream(fr, w, h, quant=quant, bitrate=bitrate, intra_period=intra)
    drec, dmbs, dw, dh = O.decode_stream(bits)
    assert (dw, dh) == (w, h) and drec.shape[0] == fr.shape[0]
    assert np.array_equal(drec, recon)
    assert list(dmbs["quant"].max(axis=1)) == list(quants)
    if quant:
        enc = O.encode_sequence(fr, w, h, quant, intra_period=intra)["mbs"]
        for i in range(fr.shape[0]):
            assert coded_equal(enc[i], dmbs[i]), f"picture {i}: records"


def test_decoder_refuses_a_damaged_stream():
    fr = synth.clip(0, 176, 144, 7, 2)
    bits = O.encode_stream(fr, 176, 144, quant=8)[0]
    with pytest.raises(ValueError):
        O.decode_stream(bits[:len(bits) // 3])
    with pytest.raises(ValueError):
        O.decode_stream(b"\xff" + bits[1:])
