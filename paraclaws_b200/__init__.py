"""paraclaws_b200: B200-native wave-propagation finite-volume step of paraCLAWs."""
