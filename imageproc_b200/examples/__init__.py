"""Programs mirroring imageproc's examples/ on the device path."""
