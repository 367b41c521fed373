"""deeprwcap_b200 — B200-native floating-random-walk transition engine."""
