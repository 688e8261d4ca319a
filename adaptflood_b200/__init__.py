"""B200-native AdaptFlood local-inertial time step."""
