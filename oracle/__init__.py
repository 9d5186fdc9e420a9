"""CPU FP64 oracle for the Pfaffian-backflow VMC hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``neuralhubbard_b200``) imports this
package.  Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may use it, and only as the checker or as the
timed CPU restatement, never as the thing that is measured on the GPU.

What it restates (reference paths relative to the ChenAo-Phys/NeuralHubbard tree):

* ``lattice``     displacement tables and minimum-image distances
                  (``code/backflow/pf_kernel.py:83-96``), hop directions of
                  ``Hubbard(U, t=[1, t'], n_neighbor=[1, 2])`` (``code/states.py:244-247``),
                  the Flip(0) @ Flip(1) @ SpinInverse() group (``code/states.py:274-279``).
* ``backflow``    ``build_wtilde`` (``pf_kernel.py:107-124``), the occupied-block gather
                  (``pf_kernel.py:156-166,371-401``) and its einsum twin
                  (``code/backflow/models.py:163-206``), the backflow CNN of the graded
                  configuration (4 periodic 3x3 layers, 32 channels, tanh-GELU) and
                  ``PfaffianBackflow.__call__`` (``models.py:208-211``).
* ``pfaffian``    batched FP64 Parlett-Reid log-Pfaffian with partial pivoting (the
                  published LTL^T algorithm of M. Wimmer, ACM TOMS 38, 30 (2012)), which is
                  what ``fermix.slogpf`` (``models.py:210``) computes.
* ``projection``  the 8 symmetry images with their fermionic reordering signs and the
                  projected amplitude.
* ``hubbard``     hop enumeration with Jordan-Wigner signs, the local energy, and a
                  Fock-space brute force of H for tiny lattices.
* ``sampler``     Philox4x32-10 counters (Salmon et al., SC'11) and the Metropolis hop
                  step, integrated autocorrelation time, block jackknife
                  (``code/measure/assemble.py:48-84``).
* ``proposal``    the learned hop-proposal CNN forward/backward (FP64), for gradient checks.
* ``resconv``     the released states' residual network (16 blocks x 64 channels,
                  ``code/backflow/models.py:319-329``), restated from its published description.
* ``port``        ctypes wrapper of ``c/nh_port.c``, the same projected amplitude compiled
                  (gcc, OpenMP): the CPU baseline of ``bench.py``, checked against the numpy code.

Parity status: the Pfaffian is pinned by known-answer tests from mathematics
(pf^2 = det, pf(B^T A B) = det(B) pf(A), block-diagonal products, brute-force expansion);
the Hamiltonian by a Fock-space brute force; the gather by its two reference formulas
(kernel order and einsum twin) agreeing.  The conventions that live inside quantax 0.4.0
and fermix 0.1.0 (``fermion_inverse_sign``, the exact Flip maps and image signs, the
projection normalisation, the residual network) cannot be executed here (no JAX in this
image); they are defined from the mathematics of the second-quantised state and the
published network description, and pinned together end to end by the released
``tpm02_L16_pfaffian`` state: its projected local energy on its own stored chains reproduces
the published E/N (``tests/test_gpu_resconv.py``).
"""
