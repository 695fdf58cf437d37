"""B200-native memetic-GA hot path for TSP (drop-in for lucasgaldinos/tsp_gpu_clean strategies)."""
