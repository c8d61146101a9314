/* Empty stand-in used when the reference CUDA kernel file is compiled as host C++ (oracle/Makefile). */
