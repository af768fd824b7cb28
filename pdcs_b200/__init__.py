"""B200-native PDHG conic solver (PDCS problem form)."""
