"""B200-native BSE kernel engine for Xatu's exciton hot path."""
