"""Learned subgrid closure: CNN kernels on BF16 tensor cores (tcgen05)."""
