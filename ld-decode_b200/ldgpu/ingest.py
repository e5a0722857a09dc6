"""Capture ingest on the GPU.

`.lds` files (DomesdayDuplicator 10-bit packed, 4 samples in 5 bytes) are
read as bytes and unpacked on the device (ldg_unpack_lds) into the signed
16-bit samples of the reference's loader (load_packed_data_4_40,
lddecode/utils.py:371-410), so a capture crosses PCIe at 1.25 bytes per
sample instead of 2."""

import numpy as np

from . import lib as L


def unpack_lds(packed, first, n, out=None, stream=None):
    """Samples [first, first + n) of a packed device buffer (torch uint8
    tensor whose byte 0 starts sample 0) as an int16 device tensor."""
    import torch
    if out is None:
        out = torch.empty(max(int(n), 1), dtype=torch.int16, device=packed.device)
    h = getattr(stream, "cuda_stream", stream) if stream is not None else torch.cuda.current_stream().cuda_stream
    L.check(L.load().ldg_unpack_lds(packed.data_ptr(), packed.numel(), int(first), int(n), out.data_ptr(),
                                    h if h else 1))
    return out[:n]


def load_packed_data_4_40(infile, sample, readlen):
    """utils.py:393-410 with the unpacking on the GPU: `readlen` samples
    from sample `sample` of an open .lds file, int16 numpy, or None when the
    file ends first."""
    import torch
    start = (sample // 4) * 5
    offset = sample % 4
    infile.seek(start)
    needed = int(np.ceil(readlen * 5 // 4)) + 5
    inbuf = infile.read(needed)
    if len(inbuf) < needed:
        return None
    dev = torch.device("cuda", torch.cuda.current_device())
    packed = torch.frombuffer(bytearray(inbuf), dtype=torch.uint8).to(dev)
    out = unpack_lds(packed, offset, readlen)
    return out.cpu().numpy()
