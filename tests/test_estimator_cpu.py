"""FP64 restatement of the DM-RS channel estimator against the reference's own outputs (the
internal FP32 frequency response and the port scalars)."""
import numpy as np

import golden_io
from fp64 import estimate_port_fp64, rel_err

BETA = float(np.float32(10 ** (3 / 20)))


def test_fp64_estimator_matches_reference_golden():
    for c in golden_io.est_cases():
        cfg = dict(nof_layers=c["nof_layers"], scaling=BETA, rb_start=c["rb_start"], nof_rb=c["nof_rb"],
                   dmrs_symbols=c["dmrs"], slot=c["slot"], n_id=c["n_id"])
        for p in range(c["ports"]):
            e = estimate_port_fp64(c["grid"], p, cfg)
            assert rel_err(c["freq"][p], e["freq"]).max() < 1e-4
            nv, epre, snr, *rsrp = c["scalars"][p]
            assert abs(nv - e["noise_var"]) / e["noise_var"] < 1e-4
            assert abs(epre - e["epre"]) / e["epre"] < 1e-4
            assert abs(snr - e["snr"]) / e["snr"] < 1e-4
            assert np.allclose(rsrp, e["rsrp"], rtol=1e-4)
