"""Helpers of the GPU tests: device buffers allocated outside torch's pool."""


class short_device_buffer:
    """A cudaMalloc'd buffer of `nbytes` (not from torch's pool, whose
    blocks sit inside larger allocations); yields its address, or None when
    the driver reports a larger extent for it than was asked for."""

    def __init__(self, nbytes):
        self.nbytes = nbytes
        self.ptr = None

    def __enter__(self):
        from cuda.bindings import driver, runtime

        err, ptr = runtime.cudaMalloc(self.nbytes)
        assert err == runtime.cudaError_t.cudaSuccess
        self.ptr = int(ptr)
        err, _, size = driver.cuMemGetAddressRange(driver.CUdeviceptr(self.ptr))
        return self.ptr if err == driver.CUresult.CUDA_SUCCESS and size == self.nbytes else None

    def __exit__(self, *exc):
        from cuda.bindings import runtime

        runtime.cudaFree(self.ptr)
