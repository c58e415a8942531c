"""Orthorhombic periodic box (gamdpy/simulation_boxes/orthorhombic.py).

The device-side minimum image, wrap and skin test are in the CUDA library;
the host functions here are plain numpy versions of the same float32
arithmetic (orthorhombic.py:43-132), used for host-side checks and the
reference's own box tests.
"""
import numpy as np


class Orthorhombic:
    """Rectangular periodic box with edge lengths ``lengths`` (float32)."""

    def __init__(self, D, lengths):
        self.D = D
        self.lengths = np.array(lengths, dtype=np.float32)
        self.len_sim_box_data = D

    def get_volume(self):
        return self.get_volume_function()(self.lengths)

    def get_volume_function(self):
        D = self.D

        def volume(sim_box):
            vol = sim_box[0]
            for i in range(1, D):
                vol *= sim_box[i]
            return vol

        return volume

    def get_dist_sq_dr_function(self):
        D = self.D

        def dist_sq_dr_function(ri, rj, sim_box, dr):
            dist_sq = np.float32(0.0)
            for k in range(D):
                dr[k] = ri[k] - rj[k]
                box_k = sim_box[k]
                dr[k] += (-box_k if 2.0 * dr[k] > +box_k else (+box_k if 2.0 * dr[k] < -box_k else 0.0))
                dist_sq = dist_sq + dr[k] * dr[k]
            return dist_sq

        return dist_sq_dr_function

    def get_dist_sq_function(self):
        D = self.D

        def dist_sq_function(ri, rj, sim_box):
            dist_sq = np.float32(0.0)
            for k in range(D):
                dr_k = ri[k] - rj[k]
                box_k = sim_box[k]
                dr_k += (-box_k if 2.0 * dr_k > +box_k else (+box_k if 2.0 * dr_k < -box_k else 0.0))
                dist_sq = dist_sq + dr_k * dr_k
            return dist_sq

        return dist_sq_function

    def get_apply_PBC(self):
        D = self.D

        def apply_PBC(r, image, sim_box):
            for k in range(D):
                if r[k] * 2.0 > +sim_box[k]:
                    r[k] -= sim_box[k]
                    image[k] += 1
                if r[k] * 2.0 < -sim_box[k]:
                    r[k] += sim_box[k]
                    image[k] -= 1

        return apply_PBC

    def get_dist_moved_sq_function(self):
        dist_sq_function = self.get_dist_sq_function()

        def dist_moved_sq_function(r_current, r_last, sim_box, sim_box_last):
            return dist_sq_function(r_current, r_last, sim_box)

        return dist_moved_sq_function

    def get_dist_moved_exceeds_limit_function(self):
        dist_sq_function = self.get_dist_sq_function()

        def dist_moved_exceeds_limit_function(r_current, r_last, sim_box, sim_box_last, skin, cut):
            return dist_sq_function(r_current, r_last, sim_box) > skin * skin * 0.25

        return dist_moved_exceeds_limit_function
