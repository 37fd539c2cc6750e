"""B200-native directional FMM matvec (Wave3d::eval of arbenson/ddfmm)."""
