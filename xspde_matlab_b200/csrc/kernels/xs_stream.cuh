// streaming-path kernels (2D/3D lattices too large for one CTA)
