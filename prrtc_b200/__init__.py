"""prrtc_b200 package (stub)."""
