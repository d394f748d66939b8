import ctypes as C, json
for v in ("0", "1", "3"):
    lib = C.CDLL(f"_work/exp/libn{v}.so")
    for n, tile in ((670, 256), (2010, 256), (2010, 192), (2010, 128)):
        ms = C.c_double()
        rc = lib.run(5000, n, 5000, 6, 5, C.byref(ms), tile)
        print(json.dumps(dict(variant={"0": "full", "1": "mma_only_sync", "3": "mma_only_nosync"}[v], n=n, tile=tile, ms=round(ms.value, 4), rc=rc, tops=round(21*2*5000*n*5000/(ms.value*1e-3)/1e12))), flush=True)
