"""pscf_b200: B200-native engine for the PSCF propagator hot path."""
