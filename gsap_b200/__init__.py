"""B200-native stochastic block partitioner (GSAP SBP path): see include/sbp.h."""
