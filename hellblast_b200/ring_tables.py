"""HEALPix ring tables (ring_tables.py:17-53 of the reference), built by the hb_ring_tables
kernel; integer tables bit-exact with the reference's build_ring_tables."""
from __future__ import annotations

import torch

from . import _lib as L
from . import ops


class HealpixRingTables:
    def __init__(self, nside: int, phi0: str = "healpix", device=None):
        nside = int(nside)
        if not (nside >= 1 and (nside & (nside - 1)) == 0):
            raise AssertionError("nside must be power of 2")  # ring_tables.py:19
        self.nside = nside
        self.Nr = 4 * nside - 1
        dev = torch.device("cuda") if device is None else torch.device(device)
        t = ops.ring_tables(nside, L.HB_PHI0_HEALPIX if phi0 == "healpix" else L.HB_PHI0_REFERENCE, dev)
        self.z_centers = t["z"]
        self.theta_centers = t["theta"]
        self.nphi = t["nphi"]
        self.phi_center0 = t["phi0"]
        self.ring_start = t["ring_start"]
        self.z_edges = t["z_edges"]
        self._wdz = t["weights_dz"]
        self.npix = 12 * nside * nside

    def weights_dz(self):
        return self._wdz

    def dump_host(self):
        return {"nside": self.nside, "Nr": self.Nr, "npix": self.npix,
                "z_centers": self.z_centers.cpu().numpy(), "theta_centers": self.theta_centers.cpu().numpy(),
                "nphi": self.nphi.cpu().numpy(), "phi_center0": self.phi_center0.cpu().numpy(),
                "ring_start": self.ring_start.cpu().numpy(), "z_edges": self.z_edges.cpu().numpy()}
