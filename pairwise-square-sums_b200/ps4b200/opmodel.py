"""Algorithmic work model of the search, frozen before any kernel tuning.

Minimum 32-bit lane-operations per event the reference counts (its stats_t counters,
exhaustive/s4.c:80-91, which depend on S only):

  pairs     5   one representation p^2+q^2: add, increment, compare, bucket
  triples  24   one representation triple: the two-class signed combine and sign tests
  sets4    80   one 4-set: six divisor-count products, two factor walks, residue set-up
  ext_cand 28   one divisor-pair candidate: ~4 products of the divisor walk + parity/mod-64 test
  ext_sqrt 80   one exact test: 128-bit square and two integer square roots

At S < 1e10 this is about 1.77e12 operations (177 per S).  achieved = ops / kernel time;
the peak it is compared with is the SMs' integer issue rate (4 warp-instructions, i.e.
128 lane-operations, per SM per clock).
"""
WEIGHTS = {"pairs": 5, "triples": 24, "sets4": 80, "ext_cand": 28, "ext_sqrt": 80}


def ops(stats: dict) -> int:
    return sum(w * int(stats[k]) for k, w in WEIGHTS.items())


# Which kernel of the two-kernel pipeline does which part of the work: the tile kernel
# (gen_jobs) enumerates representations and combines them; the extension engine
# (extend_jobs) sets up each 4-set (divisor counts, factor walks, residues) and walks and
# tests its divisor pairs.
GEN_EVENTS = ("pairs", "triples")
EXT_EVENTS = ("sets4", "ext_cand", "ext_sqrt")


def ops_split(stats: dict) -> tuple[int, int]:
    """(tile-kernel ops, engine ops) of the model above."""
    return (sum(WEIGHTS[k] * int(stats[k]) for k in GEN_EVENTS),
            sum(WEIGHTS[k] * int(stats[k]) for k in EXT_EVENTS))


def issue_peak_lane_ops(num_sms: int, sm_clock_hz: float) -> float:
    """Integer issue ceiling: 4 schedulers x 32 lanes per SM per clock."""
    return num_sms * 4 * 32 * sm_clock_hz
