"""B200-native Brownian-dynamics force-and-integrate path for MARS-MD."""
