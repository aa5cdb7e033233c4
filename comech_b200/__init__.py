"""B200-native voxel linear-elastic FE solver: drop-in for CoMech's engine solve call."""
