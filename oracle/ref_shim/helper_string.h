/* Empty stand-in for a CUDA-samples header the reference includes but does not use (oracle build only). */
