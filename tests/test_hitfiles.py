"""Hit files and filterbank readers on the CPU: the .hits encoder against the reference's
own voyager.hits bytes, the .dat table format, sigproc headers and metadata inference."""
import hashlib
import json
import os

import numpy as np
import pytest

from seticore_b200.dedoppler import DedopplerHit, FilterbankMetadata
from seticore_b200.hitfiles import (DatFileWriter, HitFileWriter, decode_hit, encode_hit, makeHitRecorder,
                                    read_hits, split_messages)
from seticore_b200.run_dedoppler import (ArrayFilterbankFile, FilReader, convertFromSigprocRaOrDec,
                                         loadFilterbankFile, write_fil)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "voyager_hits.npz")


def test_encoder_reproduces_reference_hits_file_bytes():
    g = np.load(GOLDEN)
    meta = json.loads(str(g["meta"]))
    assert len(meta) == 5
    for k, m in enumerate(meta):
        fb = dict(m["filterbank"])
        fb["data"] = g[f"data{k}"]
        layout = {"Hit": (0, 2), "Signal": tuple(m["signal"]["_layout"]), "Filterbank": tuple(fb["_layout"])}
        raw = encode_hit(m["signal"], fb, layout=layout)
        assert len(raw) == m["bytes"]
        assert hashlib.sha256(raw).hexdigest() == m["sha256"], f"message {k}"
        assert fb["sourceName"] == "Voyager1" and fb["numTimesteps"] * fb["numChannels"] == fb["data"].size


def test_reference_hits_file_decodes_when_present():
    from conftest import reference_root
    path = os.path.join(reference_root(), "data", "voyager.hits")
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    hits = read_hits(path)
    g = np.load(GOLDEN)
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == str(g["file_sha256"])
    assert [h["signal"]["index"] for h in hits] == [40] * 5
    assert [h["signal"]["driftSteps"] for h in hits] == [36, 39, 37, 38, 39]


def _meta(**kw):
    base = dict(fch1=8421.38671875, foff=-2.7939677238464355e-06, tsamp=18.253611008, coarse_channel_size=1000,
                num_timesteps=16, num_channels=4000, num_coarse_channels=4, source_name="Voyager1",
                tstart=57650.78209490741, src_raj=17.17, src_dej=12.2, telescope_id=6)
    base.update(kw)
    return FilterbankMetadata(**base)


def _hit(meta, index, steps, snr=12.5, coarse=1, power=3.0e10, beam=-1):
    return DedopplerHit.make(meta, index, steps, steps * 0.0102, snr, beam, coarse, meta.num_timesteps, power)


def test_hits_file_round_trip_current_layout(tmp_path):
    meta = _meta()
    data = np.arange(16 * 1000, dtype=np.float32).reshape(16, 1000)
    hits = [_hit(meta, 5, 3), _hit(meta, 500, -7), _hit(meta, 990, 4)]
    fn = str(tmp_path / "out.hits")
    with HitFileWriter(fn, meta) as w:
        w.recordHits(hits, data)
        assert os.path.exists(fn + ".tmp") and not os.path.exists(fn)
    assert os.path.exists(fn) and not os.path.exists(fn + ".tmp")
    got = read_hits(fn)
    assert len(got) == 3
    for h, g in zip(hits, got):
        s, f = g["signal"], g["filterbank"]
        assert (s["index"], s["driftSteps"], s["coarseChannel"], s["beam"], s["numTimesteps"]) == \
            (h.index, h.drift_steps, 1, -1, 16)
        assert s["frequency"] == h.frequency and s["driftRate"] == h.drift_rate
        assert np.float32(s["snr"]) == np.float32(h.snr) and np.float32(s["power"]) == np.float32(h.power)
        begin = max(h.lowIndex() - 40, 0)
        end = min(h.highIndex() + 40, 1000) - 1  # hit_file_writer.cpp:85 keeps the "- 1"
        assert (f["startChannel"], f["numChannels"]) == (begin, end - begin)
        assert f["fch1"] == meta.fch1 + (1000 + begin) * meta.foff
        np.testing.assert_array_equal(f["data"].reshape(16, -1), data[:, begin:end])
        assert f["sourceName"] == "Voyager1" and f["telescopeId"] == 6 and f["tstart"] == meta.tstart
        assert tuple(s["_layout"]) == (6, 0) and tuple(f["_layout"]) == (9, 2)


def test_dat_file_format(tmp_path):
    meta = _meta()
    fn = str(tmp_path / "x" / "run.dat")
    os.makedirs(os.path.dirname(fn))
    hits = [_hit(meta, 5, 3), _hit(meta, 500, -7, snr=101.25, coarse=3)]
    w = DatFileWriter(fn, meta, 4.0)
    w.recordHits(hits)
    w.close()
    lines = open(fn).read().split("\n")
    assert lines[1] == "# File ID: run.dat "
    assert lines[3] == "# Source:Voyager1"
    assert lines[4] == f"# MJD: {meta.tstart:18.12f}\tRA: 17.170000\tDEC: 12.200000"
    assert lines[5] == ("# DELTAT:  18.253611\tDELTAF(Hz):  -2.793968\tmax_drift_rate:   4.000000\t"
                        "obs_length: 292.057776")
    assert lines[7].startswith("# Top_Hit_# \tDrift_Rate \tSNR \t") and lines[7].endswith("Full_number_of_hits \t")
    row = lines[9].split("\t")
    freq = meta.fch1 + (1 * 1000 + 5) * meta.foff
    assert row[0] == "1" and row[1] == f"{3 * 0.0102:10.6f}" and row[2] == f"{12.5:10.6f}"
    assert row[3] == row[4] == row[6] == row[7] == f"{freq:14.6f}" and row[5] == "5"
    assert row[8:] == ["0.0", "0.000000", "1", "1", ""]
    assert lines[10].split("\t")[0] == "2" and lines[10].split("\t")[10] == "3"


def test_make_hit_recorder_by_suffix(tmp_path):
    meta = _meta()
    assert isinstance(makeHitRecorder(str(tmp_path / "a.dat"), meta, 1.0), DatFileWriter)
    w = makeHitRecorder(str(tmp_path / "a.hits"), meta, 1.0)
    assert isinstance(w, HitFileWriter)
    w.close()
    with pytest.raises(ValueError):
        makeHitRecorder(str(tmp_path / "a.txt"), meta, 1.0)


def test_sigproc_angles():
    assert convertFromSigprocRaOrDec(171012.0) == pytest.approx(17 + 10 / 60 + 12 / 3600)
    assert convertFromSigprocRaOrDec(-121530.5) == pytest.approx(-(12 + 15 / 60 + 30.5 / 3600))


def test_fil_round_trip_and_green_bank_inference(tmp_path):
    meta = _meta(src_raj=17.5, src_dej=-12.25)
    data = np.random.default_rng(0).random((16, 2 * 1048576), dtype=np.float32)
    fn = str(tmp_path / "g.fil")
    write_fil(fn, data, meta)
    f = loadFilterbankFile(fn)
    assert isinstance(f, FilReader)
    assert (f.num_timesteps, f.num_channels, f.coarse_channel_size, f.num_coarse_channels) == (16, 2097152, 1048576, 2)
    assert f.has_dc_spike and f.telescope_id == 6 and f.source_name == "Voyager1"
    assert f.src_raj == pytest.approx(17.5) and f.src_dej == pytest.approx(-12.25)
    assert (f.fch1, f.foff, f.tsamp, f.tstart) == (meta.fch1, meta.foff, meta.tsamp, meta.tstart)
    out = np.zeros((16, 1048576), np.float32)
    f.loadCoarseChannel(1, out)
    np.testing.assert_array_equal(out, data[:, 1048576:])
    with pytest.raises(RuntimeError):
        loadFilterbankFile(str(tmp_path / "x.h5"))


def test_metadata_inference_rules():
    a = ArrayFilterbankFile(np.zeros((16, 3 * 999424), np.float32), telescope_id=-1)
    assert (a.coarse_channel_size, a.has_dc_spike, a.num_coarse_channels) == (999424, True, 3)
    b = ArrayFilterbankFile(np.zeros((4, 2000), np.float32), coarse_channel_size=500, telescope_id=6)
    assert (b.has_dc_spike, b.num_coarse_channels) == (True, 4)
    c = ArrayFilterbankFile(np.zeros((4, 2000), np.float32), coarse_channel_size=500, telescope_id=9)
    assert c.has_dc_spike is False
    with pytest.raises(ValueError):
        ArrayFilterbankFile(np.zeros((4, 2000), np.float32))


def test_subset_metadata_and_beams():
    m = _meta(source_names=["a", "b"], ras=[1.0, 2.0], decs=[3.0, 4.0])
    assert m.getBeamSourceName(1) == "b" and m.getBeamSourceName(-1) == "Voyager1"
    assert m.getBeamRA(0) == 1.0 and m.getBeamDec(5) == 12.2
    s = m.getSubsetMetadata(1, 2, 4)
    assert s.num_channels == 1000 and s.num_coarse_channels == 1 and s.source_name == "b"
    assert s.fch1 == m.fch1 + m.foff * 1000 * 2 and s.src_raj == 2.0 and s.src_dej == 4.0
