"""Host-side storage in the reference layout for the C-ABI entry points.

HostStorage allocates the six gamera_no_storage structs of a run and the
arrays they point to (numpy, or page-locked torch CPU tensors when pinned),
so the drop-in step can be called with host buffers.
"""
import ctypes as C

import numpy as np

from . import abi

STATE = ("conserved", "old_conserved", "cell_magnetic", "old_cell_magnetic",
         "face_flux", "old_face_flux")


class HostStorage:
    """Six reference-layout storages; with scratch=False only the state
    arrays the step reads and writes are allocated (the scratch pointers of
    the struct stay NULL)."""

    def __init__(self, active, ghost, pinned=False, scratch=True):
        self.active = tuple(int(a) for a in active)
        self.ghost = int(ghost)
        self.pinned = pinned
        self.storage = (abi.Storage * abi.FACE_COUNT)()
        self._keep = []
        g = self.ghost
        ce = (self.active[0] + 2 * g, self.active[1] + 2 * g, self.active[2] + 2 * g)
        ncell = ce[0] * ce[1] * ce[2]
        self.bytes_state = 0
        for f in range(abi.FACE_COUNT):
            s = self.storage[f]
            for a in range(3):
                s.cell_extent[a] = ce[a]
            for d in range(3):
                for a in range(3):
                    s.face_extent[d][a] = ce[a] + (1 if a == d else 0)
                    s.edge_extent[d][a] = ce[a] + (0 if a == d else 1)
            s.conserved = self._alloc(5 * ncell, True)
            s.old_conserved = self._alloc(5 * ncell, True)
            s.cell_magnetic = C.cast(self._alloc(3 * ncell, True), C.POINTER(abi.Vec3))
            s.old_cell_magnetic = C.cast(self._alloc(3 * ncell, True),
                                         C.POINTER(abi.Vec3))
            if scratch:
                s.predicted_conserved = self._alloc(5 * ncell)
                s.predicted_cell_magnetic = C.cast(self._alloc(3 * ncell),
                                                   C.POINTER(abi.Vec3))
                s.hydro_rate = self._alloc(5 * ncell)
                s.maxwell_rate = C.cast(self._alloc(3 * ncell), C.POINTER(abi.Vec3))
            for d in range(3):
                fe = s.face_extent[d]
                ee = s.edge_extent[d]
                nf = fe[0] * fe[1] * fe[2]
                ne = ee[0] * ee[1] * ee[2]
                s.face_flux[d] = self._alloc(nf, True)
                s.old_face_flux[d] = self._alloc(nf, True)
                if scratch:
                    s.predicted_face_flux[d] = self._alloc(nf)
                    s.fluid_face_flux[d] = self._alloc(5 * nf)
                    s.maxwell_face_flux[d] = C.cast(self._alloc(3 * nf),
                                                    C.POINTER(abi.Vec3))
                    s.edge_emf[d] = self._alloc(ne)

    def _alloc(self, count, state=False):
        if state:
            self.bytes_state += 8 * count
        if self.pinned:
            import torch
            t = torch.zeros(count, dtype=torch.float64, pin_memory=True)
            self._keep.append(t)
            return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))
        a = np.zeros(count, dtype=np.float64)
        self._keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_double))

    def arrays(self, face):
        return abi.storage_arrays(self.storage[face])
