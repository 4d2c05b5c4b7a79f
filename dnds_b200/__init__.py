"""dnds_b200: B200-native residual-evaluation path of the DNDS compact finite-volume solver."""
