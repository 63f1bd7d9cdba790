"""Helpers for the GPU tests: run a plan through the C ABI on device buffers
(torch CUDA tensors are used only as device memory) and bring results back."""
import numpy as np

import zldsp_fft_b200 as Z


def dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t) -> np.ndarray:
    return t.cpu().numpy()


def complex_to_dev(x: np.ndarray, layout: int):
    """Batch (b, n) complex -> (ptr0, ptr1, keepalive) in the given layout."""
    if layout == Z.AOS:
        t = dev(x)
        return t.data_ptr(), None, [t]
    re, im = dev(np.ascontiguousarray(x.real)), dev(np.ascontiguousarray(x.imag))
    return re.data_ptr(), im.data_ptr(), [re, im]


def alloc_complex(b, n, layout, cdt):
    import torch
    rdt = torch.float32 if cdt == np.complex64 else torch.float64
    if layout == Z.AOS:
        t = torch.zeros((b, n, 2), dtype=rdt, device="cuda")
        return t.data_ptr(), None, [t]
    re = torch.zeros((b, n), dtype=rdt, device="cuda")
    im = torch.zeros((b, n), dtype=rdt, device="cuda")
    return re.data_ptr(), im.data_ptr(), [re, im]


def fetch_complex(keep, layout, cdt) -> np.ndarray:
    if layout == Z.AOS:
        a = host(keep[0])
        return (a[..., 0] + 1j * a[..., 1]).astype(cdt)
    return (host(keep[0]) + 1j * host(keep[1])).astype(cdt)


def run_c2c(plan, x, forward, il=Z.AOS, ol=Z.AOS):
    import torch
    b, n = x.shape
    i0, i1, ki = complex_to_dev(x, il)
    o0, o1, ko = alloc_complex(b, n, ol, x.dtype.type)
    plan.exec_device(Z.FORWARD if forward else Z.BACKWARD, il, ol, i0, i1, o0, o1, b)
    torch.cuda.synchronize()
    return fetch_complex(ko, ol, x.dtype.type)


def run_r2c(plan, x, ol=Z.AOS, sqr_mag=False):
    import torch
    b, n = x.shape
    nb = n // 2 + 1
    ti = dev(x)
    cdt = np.complex64 if x.dtype == np.float32 else np.complex128
    if sqr_mag:
        to = torch.zeros((b, nb), dtype=ti.dtype, device="cuda")
        plan.exec_device(Z.FORWARD_SQR_MAG, Z.AOS, Z.AOS, ti.data_ptr(), None, to.data_ptr(), None, b)
        torch.cuda.synchronize()
        return host(to)
    o0, o1, ko = alloc_complex(b, nb, ol, cdt)
    plan.exec_device(Z.FORWARD, Z.AOS, ol, ti.data_ptr(), None, o0, o1, b)
    torch.cuda.synchronize()
    return fetch_complex(ko, ol, cdt)


def run_c2r(plan, X, il=Z.AOS):
    import torch
    b, nb = X.shape
    n = 2 * (nb - 1)
    i0, i1, ki = complex_to_dev(X, il)
    rdt = torch.float32 if X.dtype == np.complex64 else torch.float64
    to = torch.zeros((b, n), dtype=rdt, device="cuda")
    plan.exec_device(Z.BACKWARD, il, Z.AOS, i0, i1, to.data_ptr(), None, b)
    torch.cuda.synchronize()
    return host(to)
