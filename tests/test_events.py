"""Cadence event matching on the CPU: findHit's behaviour, the ABACAD candidate rules and
the .events encoding."""
import numpy as np

from seticore_b200.dedoppler import DedopplerHit, FilterbankMetadata
from seticore_b200.events import findHit, match_events, removeZeroDriftHits
from seticore_b200.hitfiles import decode_event, encode_event, split_messages

META = FilterbankMetadata(fch1=8000.0, foff=-2.7939677e-6, tsamp=18.253611, coarse_channel_size=100000,
                          num_timesteps=16)
TSAMP = META.tsamp


def hit(index, steps, snr=20.0):
    return DedopplerHit.make(META, index, steps, steps * -0.0102, snr, -1, 0, 16, 1e10)


def keyed(hits):
    m = {h.index: h for h in hits}
    return sorted(m), m


def test_find_hit_counts_and_first_hit_past_the_range():
    a, b = hit(5, 1), hit(100, 1)
    keys, m = keyed([a, b])
    assert findHit(keys, m, 0, 10) == (1, a)
    assert findHit(keys, m, 6, 10) == (1, b)  # the first hit at or after low, even past high
    assert findHit(keys, m, 0, 200) == (2, None)
    assert findHit(keys, m, 101, 200) == (0, None)
    assert findHit([], {}, 0, 10) == (0, None)


def test_remove_zero_drift():
    assert [h.index for h in removeZeroDriftHits([hit(1, 0), hit(2, 3), hit(3, 0)])] == [2]


def _cadence(c0=40000, steps=8, gap_s=300.0):
    """Six ABACAD observations: the "on" files (0, 2, 4) see a tone starting at c0 that
    drifts `steps` channels per 15 timesteps; tstarts are gap_s apart."""
    tstarts = [i * gap_s / 86400.0 * 86400.0 for i in range(6)]
    lists = [[] for _ in range(6)]
    for i in (0, 2, 4):
        t = int(round(tstarts[i] / TSAMP))
        lists[i].append(hit(c0 + int(round(t * steps / 15.0)), steps))
    return lists, tstarts


def test_event_found_when_only_the_ons_see_it():
    lists, tstarts = _cadence()
    ev = match_events(lists, tstarts, TSAMP, 100000)
    assert len(ev) == 1
    assert [h is None for h in ev[0]] == [False, True, False, True, False, True]
    assert ev[0][0].index == 40000


def test_event_rejected_when_an_on_misses_or_an_off_sees_it():
    lists, tstarts = _cadence()
    lists[4] = []
    assert match_events(lists, tstarts, TSAMP, 100000) == []
    lists, tstarts = _cadence()
    lists[3] = [hit(40010, 8)]
    assert match_events(lists, tstarts, TSAMP, 100000) == []


def test_off_hit_anywhere_above_the_event_rejects_it():
    """find_events.cpp:205 searches offs in [low - 50, high - 50], and findHit reports the
    first hit at or after the low end wherever it lies: an off hit far above the event
    still rejects it; one below low - 50 does not."""
    lists, tstarts = _cadence()
    lists[1] = [hit(90000, 3)]
    assert match_events(lists, tstarts, TSAMP, 100000) == []
    lists, tstarts = _cadence()
    lists[1] = [hit(1000, 3)]
    assert len(match_events(lists, tstarts, TSAMP, 100000)) == 1


def test_wiggle_of_ten_channels_for_the_ons():
    """An "on" hit may sit 10 channels below its expected index, not 11; above it, the
    first hit at or after the low end counts wherever it lies (findHit)."""
    lists, tstarts = _cadence()
    lists[2][0].index -= 10
    assert len(match_events(lists, tstarts, TSAMP, 100000)) == 1
    lists, tstarts = _cadence()
    lists[2][0].index -= 11
    assert match_events(lists, tstarts, TSAMP, 100000) == []
    lists, tstarts = _cadence()
    lists[2][0].index += 500
    assert len(match_events(lists, tstarts, TSAMP, 100000)) == 1


def test_two_ons_in_range_reject():
    lists, tstarts = _cadence()
    lists[2].append(hit(lists[2][0].index + 3, 8))
    assert match_events(lists, tstarts, TSAMP, 100000) == []


def test_event_message_round_trip():
    fb = {"sourceName": "X", "fch1": 1.5, "numTimesteps": 2, "numChannels": 3, "startChannel": 7,
          "data": np.arange(6, dtype=np.float32), "coarseChannel": 4, "beam": -1}
    pairs = [({"index": 9, "driftSteps": 2, "snr": 12.0}, fb), (None, dict(fb, sourceName="OFF"))]
    raw = encode_event(pairs)
    (msg, seg), = list(split_messages(raw))
    hits = decode_event(seg)
    assert len(hits) == 2
    assert hits[0]["signal"]["index"] == 9 and hits[1]["signal"] is None
    assert hits[1]["filterbank"]["sourceName"] == "OFF"
    np.testing.assert_array_equal(hits[0]["filterbank"]["data"], np.arange(6, dtype=np.float32))
