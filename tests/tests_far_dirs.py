"""The far-field direction grid of the antenna configuration (theta 0..180, phi 0..355 degrees in
5-degree steps), shared by the fixture generator's far fields and the full-size test."""
import numpy as np


def far_dirs() -> np.ndarray:
    th = np.deg2rad(np.arange(0, 181, 5, dtype=np.float64))
    ph = np.deg2rad(np.arange(0, 360, 5, dtype=np.float64))
    t, p = np.meshgrid(th, ph, indexing="ij")
    return np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], -1).reshape(-1, 3)
