"""B200-native batched small-matrix Cholesky / LU (placeholder, filled in below)."""
