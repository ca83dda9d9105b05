"""The noise covariance (file_covmat; covmat.F90:48-591) on the oracle,
against an independent numpy statement of its formula (astro-ph/0412517
eq. 28, per pointing period):

  N^-1 = P^T C_w^-1 P - A M A^T,   A = P^T C_w^-1 F,
  M = (C_a^-1 + F^T C_w^-1 F)^-1 = Toeplitz(irfft(1 / (fcov + nshort / sigma^2)))

with the oracle's own filter spectrum (fcov), white-noise levels (sigmas)
and F^T F diagonal (nna, which trims the pointing periods) as inputs, and the file format of save_matrix: N x N native
doubles, column-major, -1 on the diagonal of unobserved pixels."""
import os

import numpy as np
import pytest

import oracle_api as O
from libmadam_b200 import synthetic as syn


def _data(seed, nnz=3, nside=8):
    cfg = syn.small_config(seed=seed, nside=nside, nsamp_obs=1 << 12, nobs=2, ndet=2,
                           temperature_only=(nnz == 1))
    return syn.to_numpy(syn.generate(cfg, nnz=nnz))


def _baselines(nsamp_iv, dnshort):
    # start_timeloop's split of an interval (parameter_control.f90:785-800)
    noba = (nsamp_iv - 1) // dnshort + 1
    lens, dn, n = [], 0.0, 0
    for _ in range(noba - 1):
        n0, dn = n, dn + dnshort
        n = int(dn + .5)
        lens.append(n - n0)
    lens.append(nsamp_iv - n)
    return np.cumsum([0] + lens)


def _segments(nna, ks, kstop, gapmin):
    """trim_interval (noise_routines.f90:763-813) applied until the interval
    is used up: runs of baselines with non-empty F^T F, split at gaps of
    gapmin empty baselines"""
    out = []
    while True:
        if not np.any(nna[ks:kstop] != 0):
            return out
        while ks < kstop and nna[ks] == 0:
            ks += 1
        while kstop > ks and nna[kstop - 1] == 0:
            kstop -= 1
        noba, gap = kstop - ks, 0
        for i in range(ks, kstop):
            if nna[i] != 0:
                gap = 0
            else:
                gap += 1
                if gap == gapmin:
                    noba = i + 1 - gap - ks
                    break
        out.append((ks, noba))
        ks += noba


def numpy_covmat(d, pars, fcov, sigmas, nna, nmap):
    ndet, nsamp = d["pixels"].shape
    npix = 12 * pars["nside_map"] ** 2
    N = npix * nmap
    nshort = int(round(pars["base_first"] * pars["fsample"]))
    nh = fcov.size // ndet
    nof = 2 * (nh - 1)
    starts = list(d["periods"]) + [nsamp]
    out = []
    for det in range(ndet):
        detw = 1 / sigmas[det] ** 2
        pix = d["pixels"][det].astype(np.int64)
        w = d["pixweights"][det].astype(np.float64).reshape(nsamp, -1)[:, :nmap]
        C = np.zeros((N, N))
        spec = 1 / (fcov[det * nh:(det + 1) * nh] + nshort * detw)
        xx = np.fft.irfft(spec, n=nof)
        edges = np.concatenate([a + _baselines(b - a, nshort)[:-1]
                                for a, b in zip(starts[:-1], starts[1:])] + [[nsamp]])
        nba = [(b - a - 1) // nshort + 1 for a, b in zip(starts[:-1], starts[1:])]
        kst = np.cumsum([0] + nba)
        nna_d = nna[det * kst[-1]:(det + 1) * kst[-1]]
        gapmin = int(60 * pars["fsample"] / nshort + 1)
        for iv in range(len(nba)):
            for k0, noba in _segments(nna_d, kst[iv], kst[iv + 1], gapmin):
                T = xx[np.abs(np.arange(noba)[:, None] - np.arange(noba)[None, :])]
                A = np.zeros((N, noba))
                for k in range(noba):
                    s = np.arange(edges[k0 + k], edges[k0 + k + 1])
                    s = s[pix[s] >= 0]
                    for c in range(nmap):
                        np.add.at(A[:, k], pix[s] * nmap + c, w[s, c])
                A *= detw
                C -= A @ T @ A.T
        good = pix >= 0
        for c1 in range(nmap):
            for c2 in range(nmap):
                np.add.at(C, (pix[good] * nmap + c1, pix[good] * nmap + c2),
                          detw * w[good, c1] * w[good, c2])
        diag = np.arange(npix) * nmap
        empty = C[diag, diag] == 0
        for c in range(nmap):
            C[diag[empty] + c, diag[empty] + c] = -1
        out.append(C)
    return out


def run_oracle_covmat(d, root, **kw):
    pars = dict(d["pars"], file_covmat=root, **kw)
    x = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.destripe(pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"],
               x["pixweights"], x["signal"], x["periods"], x["npsd"], x["psdstarts"],
               x["psdfreqs"], x["psdvals"])
    return pars


def read_covmat(root, det, N):
    a = np.fromfile("{}_{}_inv_bin.dat".format(root, det), dtype=np.float64)
    assert a.size == N * N
    return a.reshape(N, N).T  # column-major on disk


def _flag(d):
    # empty leading baselines (trimmed), a gap of more than a minute (a
    # period split in two) and a partly flagged baseline
    pix = d["pixels"]
    pix[0, :300] = -1
    pix[1, 2000:2800] = -1
    pix[0, 5000:5003] = -1
    return d


@pytest.mark.parametrize("nnz,flags", [(3, False), (1, False), (3, True)])
def test_covmat_matches_numpy_formula(tmp_path, nnz, flags):
    d = _data(161, nnz)
    if flags:
        _flag(d)
    root = str(tmp_path / "ncm")
    pars = run_oracle_covmat(d, root)
    nmap = nnz
    N = 12 * pars["nside_map"] ** 2 * nmap
    ref = numpy_covmat(d, pars, O.result("fcov"), O.result("sigmas"), O.result("nna"), nmap)
    for det, C in zip(d["dets"], ref):
        G = read_covmat(root, det, N)
        # off-diagonal blocks are mirrored (symmetrize); the diagonal blocks
        # sum their pairs in one order, symmetric to rounding
        assert np.abs(G - G.T).max() <= 1e-13 * np.abs(G).max()
        assert np.abs(G - C).max() <= 1e-9 * np.abs(C).max()
    # unobserved pixels carry the -1 sentinel, observed ones a positive diagonal
    hits = O.result("hits")
    dg = np.diag(read_covmat(root, d["dets"][0], N)).reshape(-1, nmap)[:, 0]
    assert np.all(dg[hits == 0] == -1)


def test_existing_file_is_skipped_and_map_is_binned(tmp_path):
    d = _data(162)
    root = str(tmp_path / "ncm")
    marker = "{}_{}_inv_bin.dat".format(root, d["dets"][1])
    with open(marker, "wb") as f:
        f.write(b"keep")
    run_oracle_covmat(d, root)
    assert open(marker, "rb").read() == b"keep"
    assert os.path.getsize("{}_{}_inv_bin.dat".format(root, d["dets"][0])) > 4
    # write_covmat replaces the solve: no baselines, the map is the binned map
    assert np.all(O.result("aa") == 0)
    np.testing.assert_array_equal(O.result("map"), O.result("binmap"))


def _covmat_rank(rank, world, root):
    import oracle_api as O
    import shard_util as SU
    d = _data(163)
    N = 12 * d["pars"]["nside_map"] ** 2 * 3
    O.set_comm(0, 1, None)
    run_oracle_covmat(d, "{}_full{}".format(root, rank))
    mine = SU.shard_time(d, rank, world)
    O.set_comm(rank, world, SU.gloo_allreduce)
    run_oracle_covmat(mine, root + "_shard")
    O.set_comm(0, 1, None)
    if rank == 0:
        for det in d["dets"]:
            a = read_covmat(root + "_shard", det, N)
            b = read_covmat("{}_full{}".format(root, rank), det, N)
            assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_ranks_sum_their_matrices(tmp_path):
    # each rank holds one pointing period of every detector; save_matrix
    # adds the ranks' matrices (covmat.F90:282-318) and rank 0 writes
    import shard_util as SU
    SU.run_ranks(_covmat_rank, 2, (str(tmp_path / "ncm"),))
