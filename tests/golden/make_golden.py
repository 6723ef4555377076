"""Generate the golden fixtures in this directory from the reference's own
host code (compiled by oracle/build_ref.sh from the reference tree).

Each ``*.npz`` holds a QC int4 input ``qc`` [batch, N, K] (uint8) and the
reference's packed lower triangles ``tri`` [batch, N(N+1)/2, 2]:

* herk_int4_small / herk_int4_medium: the shapes of the reference's CTest
  cases herk_int4_small (64 x 128 x 2) and herk_int4_medium (128 x 256 x 4)
  (cutlass_interface/CMakeLists.txt:833-900), input drawn exactly as
  test_herk_int4.cu:313-321 draws it (std::mt19937(42), uniform ints in
  [-7, 7], Re then Im), output from the reference's cpu_herk (:51-70).
* herk_batch_first_rawbytes: 32 x 32 x 32 arbitrary bytes (every QC code,
  negative zero included), output from the reference's cpu_herk_batch_first
  (tests/visibility_pipeline_test.cpp:136-168), the oracle of its
  CutlassHerkCorrectnessTest shape (:1188-1262).
* herk_edge_*: ragged shapes (N, K not multiples of the tile sizes, N = 1,
  K = 1) and the all-(+-7) adversarial input, from cpu_herk.
* ftd/ftd_tacp_*.npz: raw packet-ordered QC bytes [t][ant][chan][pol] and the
  per-batch triangles of the reference's cpu_herk_ftd
  (tests/visibility_pipeline_test.cpp:55-96), batch b = (chan*n_pol + pol)
  *n_time_inner + ti.

Run from the repository root: ``python tests/golden/make_golden.py``.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def ref_gen(seed, n):
    L = oracle.ref_lib()
    qc = np.empty(n, dtype=np.uint8)
    L.ref_gen_int4(seed, n, qc.ctypes.data_as(oracle._u8p))
    return qc


def save(name, qc, N, K, batch, tri):
    assert np.all(tri == np.rint(tri)), name
    np.savez_compressed(os.path.join(OUT, name + ".npz"), qc=qc.reshape(batch, N, K),
                        tri=tri.astype(np.int32), N=N, K=K, batch=batch)
    print(name, qc.size, "bytes in,", tri.shape)


def main():
    if oracle.ref_lib() is None and oracle.build_ref() is None:
        raise SystemExit("reference host code could not be built")
    oracle.ref_lib()
    for name, (N, K, batch) in {"herk_int4_small": (64, 128, 2),
                                "herk_int4_medium": (128, 256, 4)}.items():
        qc = ref_gen(42, N * K * batch)
        save(name, qc, N, K, batch, oracle.ref_cpu_herk(qc, N, K, batch))

    # raw bytes through the batch-first reference correlator
    N, K, batch = 32, 32, 32
    qc = np.random.default_rng(1234).integers(0, 256, size=N * K * batch, dtype=np.uint8)
    tri = np.empty((batch, N * (N + 1) // 2, 2), dtype=np.float32)
    oracle.ref_lib().ref_cpu_herk_batch_first(qc.ctypes.data_as(oracle._u8p), N, K, batch,
                                              tri.ctypes.data_as(oracle._f32p))
    save("herk_batch_first_rawbytes", qc, N, K, batch, tri)

    rng = np.random.default_rng(99)
    for (N, K, batch) in [(1, 1, 1), (7, 5, 2), (129, 65, 3), (200, 300, 1)]:
        re, im = oracle.gaussian_int4(rng, (batch, N, K))
        qc = oracle.encode_qc(re, im)
        save(f"herk_edge_n{N}_k{K}_b{batch}", qc, N, K, batch, oracle.ref_cpu_herk(qc, N, K, batch))

    # raw packet-ordered input through the reference's cpu_herk_ftd
    os.makedirs(os.path.join(OUT, "ftd"), exist_ok=True)
    for (n_ant, n_chan, n_pol, n_ti, K) in [(24, 3, 2, 2, 48), (37, 2, 2, 1, 70)]:
        n_time = K * n_ti
        raw = np.random.default_rng(n_ant * 100 + K).integers(
            0, 256, size=n_time * n_ant * n_chan * n_pol, dtype=np.uint8)
        nb = n_chan * n_pol * n_ti
        tri = np.stack([oracle.ref_cpu_herk_ftd(raw, b, n_ant, n_chan, n_pol, n_ti, n_time)
                        for b in range(nb)])
        name = f"ftd_tacp_a{n_ant}_c{n_chan}_p{n_pol}_ti{n_ti}_k{K}"
        assert np.all(tri == np.rint(tri)), name
        np.savez_compressed(os.path.join(OUT, "ftd", name + ".npz"), raw=raw,
                            tri=tri.astype(np.int32), n_ant=n_ant, n_chan=n_chan, n_pol=n_pol,
                            n_time_inner=n_ti, n_time=n_time)
        print(name, raw.size, "bytes in,", tri.shape)

    # adversarial: every sample +-7 in both parts (largest sums, all sign mixes)
    N, K, batch = 160, 256, 1
    s = rng.integers(0, 2, size=(2, batch, N, K)) * 2 - 1
    qc = oracle.encode_qc(7 * s[0], 7 * s[1])
    save("herk_edge_pm7_n160_k256", qc, N, K, batch, oracle.ref_cpu_herk(qc, N, K, batch))


if __name__ == "__main__":
    main()
