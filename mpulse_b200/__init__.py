"""B200-native implementation of MPulse's time-stepping hot path."""
