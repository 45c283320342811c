// adjoint kernels (placeholder until the adjoint lands)
