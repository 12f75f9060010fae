"""Seeded polar-coded UCI cases shared by the CPU and GPU tests: messages of 12 to 1706 bits
encoded by the reference's polar pieces (oracle._ref), sent as BPSK over AWGN and quantised to
int8 soft bits. The (A, E) pairs cover CRC6 and CRC11, parity-check bits with and without the
minimum-weight one, shortening, puncturing above and below 3N/4, repetition, one and two
codeblocks, the odd split with its filler bit, and the largest message."""
import numpy as np

# (A, E): message bits, rate-matched soft bits.
SIZES = [(12, 40), (12, 300), (15, 48), (19, 60), (20, 64), (20, 100), (30, 100), (40, 170), (64, 150),
         (100, 400), (200, 600), (300, 1000), (359, 1500), (360, 1088), (361, 2000), (500, 3000),
         (1000, 1500), (1013, 4000), (1706, 8000)]
SNR_DB = [6.0, 0.0]


def cases(ref, seed=0):
    """[(A, soft bits int8, message bits)] for every size at both SNRs."""
    rng = np.random.default_rng(seed)
    out = []
    for A, E in SIZES:
        for snr in SNR_DB:
            msg = rng.integers(0, 2, A).astype(np.uint8)
            enc = ref.uci_polar_encode(msg, E)
            sigma = 10.0 ** (-snr / 20.0)
            y = (1.0 - 2.0 * enc) + sigma * rng.standard_normal(E)
            llr = np.clip(np.round(2.0 * y / sigma ** 2 * 4.0), -120, 120).astype(np.int8)
            out.append((A, llr, msg))
    return out
