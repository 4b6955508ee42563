"""Learned Lanczos start vector: compression of ground states onto proton x neutron
sub-blocks, the interaction sweep that produces training data with the GPU solver, the
network (trained by libnsx's own CUDA kernels) and the start vector built from it."""
