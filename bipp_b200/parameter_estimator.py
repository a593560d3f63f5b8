"""Energy-level intervals from eigenvalue spectra.

Same interface and semantics as the reference's python/bipp/parameter_estimator.py:18-105
(k-means with random_state 42 on log or linear eigenvalues, intervals at centroid
midpoints). Used to calibrate the levels of a synthesis run from the eigenvalues of
its first steps.
"""
from __future__ import annotations

import numpy as np


def centroid_to_intervals(centroid=None, d_min=0.0, d_max=float(np.finfo("f").max)):
    if centroid is None or centroid.size <= 1:
        return np.array([[d_min, d_max]])
    intervals = np.empty((centroid.size, 2))
    order = np.argsort(centroid)
    srt = centroid[order]
    for i in range(centroid.size):
        idx = order[i]
        intervals[i, 0] = d_min if idx == 0 else (srt[idx] + srt[idx - 1]) / 2
        intervals[i, 1] = d_max if idx == centroid.size - 1 else (srt[idx] + srt[idx + 1]) / 2
    return intervals


def infer_intervals(n_level, sigma, cluster_func, d_min, d_max, d_all):
    import sklearn.cluster as skcl

    if cluster_func == "log" and d_min < 0:
        raise ValueError(f'Cluster function "log" requires non-negative minimum eigenvalue restriction. Got {d_min}')
    d_all = np.array(d_all).flatten()
    d_all = d_all[d_all != 0.0]
    d_all = d_all[(d_all >= d_min) & (d_all <= d_max)]
    if 0 <= sigma < 1:
        n_remove = int((1 - sigma) * d_all.shape[0])
        if n_remove <= d_all.shape[0]:
            d_all = np.sort(d_all)[0:-n_remove]
    d_all = d_all.reshape(-1, 1)
    if cluster_func == "log":
        km = skcl.KMeans(n_clusters=n_level, random_state=42).fit(np.log(d_all))
        centroid = np.sort(np.exp(km.cluster_centers_)[:, 0])[::-1]
    elif cluster_func == "none":
        km = skcl.KMeans(n_clusters=n_level, random_state=42).fit(d_all)
        centroid = np.sort(km.cluster_centers_[:, 0])[::-1]
    else:
        raise ValueError(f'Unknown cluster function "{cluster_func}".')
    return centroid_to_intervals(centroid, d_min, d_max)
