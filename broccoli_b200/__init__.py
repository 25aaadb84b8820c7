"""broccoli_b200 -- B200-native registration and filtering hot path of BROCCOLI."""
