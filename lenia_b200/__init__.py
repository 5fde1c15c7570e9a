"""B200-native 3D Flow Lenia step."""
