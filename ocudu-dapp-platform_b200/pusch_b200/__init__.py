"""pusch_b200: B200-native (sm_100a) PUSCH receive path behind the reference's PHY interfaces.

Modules
  _native  ctypes binding of the C ABI (include/pusch_b200.h)
  ldpc     LdpcDecoder / LdpcBatchDecoder (ocudu::ldpc_decoder and the batch decoder interface)
  codec    transmit-side CRC and LDPC encoding for the seeded simulator
  sim      seeded synthetic workloads
"""
__all__ = ["_native", "ldpc", "codec", "sim"]
