"""The reference encoder's application on the B200 core: YUV 4:2:0 files in,
an H.261 bitstream and the reconstruction out, one line of statistics per
picture (src/h261_main.c:95-327).

    python -m h261enc_cuda_b200.app in.yuv out.h261 recon.yuv \\
        [--width 352 --height 288] [--bitrate 512000 | --quant Q] [--intra-period N]

What the reference's main does, kept here:

* planar 4:2:0 pictures read back to back, Y then Cb then Cr
  (h261_main.c:178-184); the stream ends at the first short read;
* the first picture is intra, the rest inter, unless an intra period is
  given (the reference has none);
* CBR rate control at 512 kbit/s from QUANT 10 with a one-second VBV
  (h261_main.c:165), or a fixed QUANT;
* the bitstream file is every picture's bytes in order (h261_main.c:253-255)
  and the reconstruction file every reconstructed picture (:262-264);
* per picture: QUANT, rate-control cost, bytes, PSNR of Y, Cb, Cr and time;
  at the end the mean PSNRs, kbit/s at 29.97 Hz and pictures per second.

The encoding, the bitstream and the PSNR are computed on the device
(motion search to bitstream in the encode and bitstream kernels; squared
errors summed by the encode kernel); this module only moves files.
"""
from __future__ import annotations

import argparse
import sys
import time
from dataclasses import dataclass
from typing import Callable, Iterator, List, Optional

import numpy as np

from .engine import Engine


def frame_bytes(width: int, height: int) -> int:
    return width * height * 3 // 2


def read_yuv(path: str, width: int, height: int, max_frames: Optional[int] = None) -> np.ndarray:
    """Every whole picture of a planar 4:2:0 file as (n, W*H*3/2) uint8; a
    trailing partial picture is ignored, as the reference's read loop does."""
    data = np.fromfile(path, np.uint8)
    fs = frame_bytes(width, height)
    n = data.size // fs
    if max_frames is not None:
        n = min(n, max_frames)
    return data[:n * fs].reshape(n, fs)


def iter_yuv(path: str, width: int, height: int) -> Iterator[np.ndarray]:
    """The pictures of a planar 4:2:0 file one at a time (no whole-file read)."""
    fs = frame_bytes(width, height)
    with open(path, "rb") as f:
        while True:
            b = f.read(fs)
            if len(b) < fs:
                return
            yield np.frombuffer(b, np.uint8)


def write_yuv(path: str, frames) -> None:
    with open(path, "wb") as f:
        for fr in frames:
            f.write(np.ascontiguousarray(fr, np.uint8).tobytes())


@dataclass
class PictureStats:
    frame: int
    quant: int
    cost: int          # the rate control's picture cost: max(sum of MB costs, 100 per MB)
    size: int          # bytes
    psnr: tuple        # (Y, Cb, Cr) dB
    time_ms: float

    def line(self) -> str:
        """The reference's per-picture line (h261_main.c:268-274)."""
        return (f"frame {self.frame:04d}, quant={self.quant}, cost={self.cost}, size={self.size}, "
                f"ypsnr={self.psnr[0]:f}, cbpsnr={self.psnr[1]:f}, crpsnr={self.psnr[2]:f}, "
                f"time={self.time_ms:.3f}ms")


def encode_file(in_path: str, bits_path: str, recon_path: str, width: int = 352, height: int = 288,
                quant: int = 0, bitrate: int = 512000, intra_period: int = 0, denoise: int = 5, device: int = 0,
                log: Optional[Callable[[str], None]] = print) -> List[PictureStats]:
    """Encode a YUV file the way the reference's main does; quant=0 selects
    the CBR rate control at `bitrate` bit/s."""
    stats: List[PictureStats] = []
    nmb = (width // 16) * (height // 16)
    t_all = time.perf_counter()
    with Engine(device=device, max_sessions=1, levels_to_host=0) as e, \
            open(bits_path, "wb") as fbits, open(recon_path, "wb") as frec:
        sid = e.open(width, height, quant if quant > 0 else 10, intra_period=intra_period, denoise=denoise,
                     bitstream=1, rate_control=0 if quant > 0 else 1, bitrate=bitrate if quant <= 0 else 0, psnr=1)
        for i, fr in enumerate(iter_yuv(in_path, width, height)):
            t0 = time.perf_counter()
            e.submit_frame(sid, fr)
            e.step()
            e.sync()
            r = e.result(sid)
            if r.bits is None:
                raise RuntimeError(f"picture {i}: no bitstream (status {r.bits_status})")
            fbits.write(r.bits)
            for plane in e.recon(sid):
                frec.write(plane.tobytes())
            cost = max(int(r.mbs["cost"].sum()), nmb * 100)
            st = PictureStats(i, r.quant, cost, len(r.bits), r.psnr, (time.perf_counter() - t0) * 1e3)
            stats.append(st)
            if log:
                log(st.line())
    elapsed = time.perf_counter() - t_all
    if log and stats:
        n = len(stats)
        mean = [sum(s.psnr[c] for s in stats) / n for c in range(3)]
        total = sum(s.size for s in stats)
        log(f"PSNR Mean: {mean[0]:f}, {mean[1]:f}, {mean[2]:f}")
        log(f"{total * 8 / (n / 0.02997):f} kBit/s, {n / elapsed:f} fps")
    return stats


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("input")
    ap.add_argument("bitstream")
    ap.add_argument("recon")
    ap.add_argument("--width", type=int, default=352)
    ap.add_argument("--height", type=int, default=288)
    ap.add_argument("--quant", type=int, default=0, help="fixed QUANT 1..31 (default: CBR rate control)")
    ap.add_argument("--bitrate", type=int, default=512000)
    ap.add_argument("--intra-period", type=int, default=0)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    encode_file(a.input, a.bitstream, a.recon, a.width, a.height, a.quant, a.bitrate, a.intra_period,
                device=a.device)
    return 0


if __name__ == "__main__":
    sys.exit(main())
