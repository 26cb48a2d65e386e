"""A device array with the small surface the reference's callers use on numba device arrays (``copy_to_host``,
``shape``, ``dtype``, ``size``, ``__cuda_array_interface__``), backed by a torch tensor.  ``numba.cuda.as_cuda_array``
and ``torch.as_tensor`` both accept it without a copy."""
import numpy as np


class DeviceArray:
    __slots__ = ("tensor",)

    def __init__(self, tensor):
        self.tensor = tensor

    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def size(self):
        return int(self.tensor.numel())

    @property
    def dtype(self):
        return np.dtype(str(self.tensor.dtype).replace("torch.", ""))

    @property
    def __cuda_array_interface__(self):
        return self.tensor.__cuda_array_interface__

    def copy_to_host(self):
        return self.tensor.cpu().numpy()

    def reshape(self, *shape):
        return DeviceArray(self.tensor.reshape(*shape))

    def __len__(self):
        return int(self.tensor.shape[0])

    def __repr__(self):
        return f"DeviceArray(shape={self.shape}, dtype={self.dtype})"
