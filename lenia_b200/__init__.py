"""B200-native 3D Flow Lenia step: the Python mirror of the C ABI (worlds,
batches), marching-cubes meshing, grid statistics and labels, and the
proposal network."""
