"""FIR-B200: FIR's projection and reconstruction path on NVIDIA B200 (sm_100a)."""
