"""A run sharded over two ranks (collect_map / collect_cc / collect_hits and
the inner products reduced across ranks, as the reference's MPI layer does)
gives the maps, hits and baselines of the single-rank run on all the data:
the oracle on two gloo ranks, sharded by detector and, as the reference's
ranks hold time slices of every detector, by time (where the leakage
matrices, one collective per detector, need every rank to hold the same
detectors)."""
import numpy as np

import shard_util as SU


def _args(pars, x):
    return (pars, x["dets"], x["detweights"], x["timestamps"], x["pixels"], x["pixweights"],
            x["signal"], x["periods"], x["npsd"], x["psdstarts"], x["psdfreqs"], x["psdvals"])


def _rank(rank, world, extra):
    import oracle_api as O
    from libmadam_b200 import synthetic as syn
    d = syn.to_numpy(syn.generate(syn.small_config(seed=101)))
    extra = dict(extra)
    subsets = extra.pop("subsets", False)
    pars = dict(d["pars"], **extra)
    if subsets:
        t = d["timestamps"]
        pars.update(bin_subsets=True, survey=["hm1 : {} - {}".format(t[0], t[len(t) // 2])],
                    detset=["AB : det000, det001"], write_leakmatrix=True)
    full = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    O.set_comm(0, 1, None)
    O.destripe(*_args(pars, full))
    ref = {k: O.result(k) for k in ("map", "binmap", "hits", "mask", "aa")}
    ref_it = O.scalars()["noiter"]
    if subsets:
        tab = O.result("subsets").reshape(-1, 4)
        ref_sub = {n: O.result(n) for k in range(len(tab))
                   for n in ("subset_binmap:%d" % k, "subset_hits:%d" % k)}
        ref_leak = O.result("leakmatrix:0")
    by_time = subsets
    mine = SU.shard_time(d, rank, world) if by_time else SU.shard(d, rank, world)
    O.set_comm(rank, world, SU.gloo_allreduce)
    O.destripe(*_args(pars, mine))
    O.set_comm(0, 1, None)
    np.testing.assert_array_equal(O.result("hits"), ref["hits"])
    np.testing.assert_array_equal(O.result("mask"), ref["mask"])
    for k in ("map", "binmap"):
        np.testing.assert_allclose(O.result(k), ref[k], rtol=0,
                                   atol=1e-9 * np.abs(ref[k]).max())
    assert O.scalars()["noiter"] == ref_it
    ndet = len(d["dets"])
    if by_time:
        np.testing.assert_array_equal(
            mine["pixels"], full["pixels"].reshape(ndet, -1)[:, slice(*mine["span"])])
    else:
        noba = ref["aa"].size // ndet
        aa = ref["aa"].reshape(ndet, noba)[mine["mine"]].reshape(-1)
        np.testing.assert_allclose(O.result("aa"), aa, rtol=0, atol=1e-9 * np.abs(aa).max())
        # the pixels each rank gets back are its own, edited as a lone run edits them
        np.testing.assert_array_equal(mine["pixels"].reshape(-1),
                                      full["pixels"].reshape(ndet, -1)[mine["mine"]].reshape(-1))
    if subsets:
        np.testing.assert_array_equal(O.result("subsets"), tab.reshape(-1))
        for n, v in ref_sub.items():
            np.testing.assert_allclose(O.result(n), v, rtol=0, atol=1e-9 * max(np.abs(v).max(), 1))
        np.testing.assert_allclose(O.result("leakmatrix:0"), ref_leak, rtol=0, atol=1e-9)


def test_two_ranks_match_one():
    SU.run_ranks(_rank, 2, (dict(),))


def test_two_ranks_with_subsets_and_no_filter():
    SU.run_ranks(_rank, 2, (dict(subsets=True, kfilter=False, diagfilter=0.5),))


def test_two_ranks_with_file_spectrum(tmp_path):
    """Every rank reads the spectrum file for the detectors it holds
    (get_spectrum_file, noise_routines.f90:600-634); the sharded run still
    gives the lone run's maps and baselines."""
    from libmadam_b200 import synthetic as syn
    from test_oracle_spectrum import _table, _write
    d = syn.to_numpy(syn.generate(syn.small_config(seed=101)))
    freq, psd, sig = _table(d)
    path = tmp_path / "spec.txt"
    _write(path, list(d["dets"]), sig, freq, psd)
    SU.run_ranks(_rank, 2, (dict(file_spectrum=str(path)),))
