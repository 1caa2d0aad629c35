"""B200-native conditional-block contraction and exact free-bit sampling."""
