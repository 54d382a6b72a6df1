"""CPU FP64 oracle for the OpenAtom Car-Parrinello electronic step.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package (``openatom_b200``)
imports, links or executes anything under ``oracle/``; only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` use it, and there only as the checker / the timed CPU baseline.

Every routine restates the reference arithmetic of OpenAtom (UIUC-PPL/OpenAtom)
and cites the reference ``file:line`` it follows.  Parity pins:

* the G-vector layout (``layout.py``) is checked bit-exact against the
  reference's own ``flip_data_set`` / ``get_chareG_line_prms`` / ``sort_commence``
  compiled from their sources under ``oracle/_ref`` (``oracle/build_ref.sh``), and
  against the committed fixtures in ``tests/golden``;
* the Ortho Schulz iteration (``ortho.py``) is checked against the reference's
  ``CPORTHOG::get_iter_Tmat`` compiled from ``cp_lowdin.C`` under ``oracle/_ref``;
* the EES non-local pass (``ees.py``: b(G) weights, spline look-up, atom
  B-splines, projector, Z matrix, energy, atom and psi forces, NL grid size)
  is checked against the reference's ``cp_ees_nonlocal.C`` and
  ``set_cp_ewald.C`` routines compiled from their sources under ``oracle/_ref``
  (``ref_ees.cpp`` fills the PINY singletons they read);
* FFT, density, V.psi, XC, Hartree and integrator arithmetic have no
  golden vectors in the reference (its regression datasets are external and
  absent), so they are pinned by mathematical identities (Parseval, electron
  count, adjointness of the forward/backward transforms, finite differences
  of the energy) in ``tests/`` -- parity for those pieces is *unpinned* by
  reference outputs.
"""
