"""B200 engine for DENSE's deterministic delay-differential simulation.

Modules (none is imported here; each loads its native library on first use):

* ``engine`` -- the C ABI of one model's engine library through ctypes:
  ``ParameterSet``, ``Analysis``, ``Batch`` (create, run, read), ``plan``.
* ``tissue``, ``csvio``, ``report`` -- DENSE's default tissue and graph
  CSR, its CSV tokenizer, and its analysis CSV text.
* ``workloads`` -- the seeded synthetic inputs of the benchmark
  configurations.
* ``mixed``, ``autotune`` -- uneven batches of several models in one CUDA
  graph, and the per-bucket schedule tuner.
* ``sharding`` -- sets over several GPUs by cost, one gather at the end.
* ``surrogate``, ``search``, ``search_run``, ``distributed`` -- the MLP on
  the tensor-core kernels, surrogate-screened parameter search and SRES,
  and their multi-GPU forms.
* ``precision_check`` -- FP32+Kahan against FP64 per configuration.
* ``build``, ``models`` -- compiling the engine, CLI and surrogate
  libraries for sm_100a from the DENSE model headers.
"""
