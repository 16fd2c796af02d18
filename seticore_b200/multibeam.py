"""Searching beamformer output in place (beamforming_pipeline.cpp:200-263).

A MultibeamBuffer holds [beam][time][channel] float32 power on the device
(multibeam_buffer.h:14-56).  The reference copies each (beam, coarse channel) region into
a separate FilterbankBuffer (MultibeamBuffer::copyRegionAsync, multibeam_buffer.cu:65-76)
and searches it; here a region is a strided view (row stride = the buffer's channel
count), which the search reads directly, and all coherent (beam, coarse channel) regions
of a band go to the device in one batched call.  The incoherent beam then adds its power
to each coarse channel's hits (Dedopplerer::addIncoherentPower), as in the reference.
"""
from typing import Dict, List, Optional

from .dedoppler import Dedopplerer, FilterbankBuffer, FilterbankMetadata


class MultibeamBuffer:
    def __init__(self, num_beams: int, num_timesteps: int, num_channels: int, device="cuda", data=None):
        import torch
        self.num_beams, self.num_timesteps, self.num_channels = num_beams, num_timesteps, num_channels
        self.data = data if data is not None else torch.zeros((num_beams, num_timesteps, num_channels),
                                                              dtype=torch.float32, device=device)
        assert tuple(self.data.shape) == (num_beams, num_timesteps, num_channels)

    def getBeam(self, beam: int) -> FilterbankBuffer:
        """multibeam_buffer.cu: a view of one beam."""
        return FilterbankBuffer(self.num_timesteps, self.num_channels, data=self.data[beam])

    def region(self, beam: int, channel_offset: int, width: int):
        """[num_timesteps][width] view of one beam starting at channel_offset: what
        copyRegionAsync copies (multibeam_buffer.cu:65-76), without the copy."""
        return self.data[beam, :, channel_offset:channel_offset + width]

    def zeroAsync(self) -> None:
        self.data.zero_()


def search_band(dedopplerer: Dedopplerer, multibeam: MultibeamBuffer, metadata: FilterbankMetadata, band: int,
                coarse_channels_per_band: int, max_drift: float, snr: float, hit_recorder=None,
                stream=None) -> List:
    """The per-band search of BeamformingPipeline::findHits (beamforming_pipeline.cpp:200-263):
    every coherent beam's coarse channels are searched (min_drift 0, as there), hits are
    recorded beam by beam, then the incoherent beam fills incoherent_power of each coarse
    channel's hits.  Returns the band's hits ordered by coarse channel, each coarse
    channel's hits in the order they were found (the reference's map iteration)."""
    fft_size = dedopplerer.num_channels
    per_cc: Dict[int, List] = {}
    coherent = [b for b in range(multibeam.num_beams) if metadata.isCoherentBeam(b)]
    jobs = [(b, lc) for b in coherent for lc in range(coarse_channels_per_band)]
    for k0 in range(0, len(jobs), 64):
        part = jobs[k0:k0 + 64]
        inputs = [multibeam.region(b, lc * fft_size, fft_size) for b, lc in part]
        res = dedopplerer.search_batch(inputs, metadata, [b for b, _ in part],
                                       [band * coarse_channels_per_band + lc for _, lc in part],
                                       max_drift, 0.0, snr, stream=stream)
        for (b, lc), hits, x in zip(part, res, inputs):
            cc = band * coarse_channels_per_band + lc
            per_cc.setdefault(cc, []).extend(hits)
            if hit_recorder is not None and hits:
                hit_recorder.recordHits(hits, x)
    for b in range(multibeam.num_beams):
        if metadata.isCoherentBeam(b):
            continue
        for lc in range(coarse_channels_per_band):
            cc = band * coarse_channels_per_band + lc
            hits = per_cc.setdefault(cc, [])
            dedopplerer.addIncoherentPower(multibeam.region(b, lc * fft_size, fft_size), hits, stream=stream)
    out = []
    for cc in sorted(per_cc):
        out.extend(per_cc[cc])
    return out
