"""Python mirror of the reference's Encoder interface on top of librsgpu.so.

    enc = New(10, 4)                     # reedsolomon.New(10, 4)
    enc.Encode(shards)                   # shards: 14 CUDA uint8 tensors
    ok = enc.Verify(shards)
    shards[3] = None                     # a missing shard, like a nil slice
    enc.Reconstruct(shards)              # fills shards[3] in place

Shards are 1-D contiguous torch.uint8 tensors.  CUDA tensors run the device
path; CPU tensors / numpy arrays run the host path (PCIe copies inside the
library).  Errors raise the exception named after the reference's sentinel
error (ErrTooFewShards, ErrShardSize, ...).
"""
import ctypes

import numpy as np
import torch

from . import _lib as L

RS_CODEC_CLASSIC, RS_CODEC_LEOPARD16, RS_CODEC_LEOPARD8 = 0, 1, 2
_MATRIX = {"default": 0, "cauchy": 1, "par1": 2, "jerasure": 3}


class RSError(Exception):
    code = None


def _err(name, code):
    return type(name, (RSError,), {"code": code})


ErrTooFewShards = _err("ErrTooFewShards", -1)
ErrShardNoData = _err("ErrShardNoData", -2)
ErrShardSize = _err("ErrShardSize", -3)
ErrInvalidShardSize = _err("ErrInvalidShardSize", -4)
ErrInvShardNum = _err("ErrInvShardNum", -5)
ErrMaxShardNum = _err("ErrMaxShardNum", -6)
ErrNotSupported = _err("ErrNotSupported", -7)
ErrInvalidInput = _err("ErrInvalidInput", -8)
ErrReconstructRequired = _err("ErrReconstructRequired", -9)
ErrSingular = _err("ErrSingular", -10)
ErrNotSquare = _err("ErrNotSquare", -11)
ErrShortData = _err("ErrShortData", -12)
ErrReconstructMismatch = _err("ErrReconstructMismatch", -13)
CudaError = _err("CudaError", -100)
ErrNoMem = _err("ErrNoMem", -101)
ErrTimeout = _err("ErrTimeout", -102)
ErrNoDevice = _err("ErrNoDevice", -103)
_BY_CODE = {c.code: c for c in (ErrTooFewShards, ErrShardNoData, ErrShardSize, ErrInvalidShardSize,
                                ErrInvShardNum, ErrMaxShardNum, ErrNotSupported, ErrInvalidInput,
                                ErrReconstructRequired, ErrSingular, ErrNotSquare, ErrShortData, ErrReconstructMismatch,
                                CudaError, ErrNoMem,
                                ErrTimeout, ErrNoDevice)}


def check(rc):
    if rc != 0:
        lib = L.lib()
        msg = lib.rsgpu_status_string(rc).decode()
        detail = lib.rsgpu_last_error().decode()
        exc = _BY_CODE.get(rc, RSError)
        raise exc("%s%s" % (msg, (": " + detail) if detail and rc <= -100 else ""))
    return rc


# ---- options (options.go) ---------------------------------------------------
def _opt(**kv):
    def apply(o):
        o.update(kv)
    return apply


def WithCauchyMatrix():
    return _opt(matrix="cauchy")


def WithPAR1Matrix():
    return _opt(matrix="par1")


def WithJerasureMatrix():
    return _opt(matrix="jerasure")


def WithFastOneParityMatrix():
    return _opt(fast_one_parity=1)


def WithCustomMatrix(rows):
    return _opt(custom=np.asarray(rows, dtype=np.uint8))


def WithLeopardGF16(enabled=True):
    return _opt(leopard=1 if enabled else 0)


def WithLeopardGF(enabled=True):
    return _opt(leopard=2 if enabled else 0)


def WithInversionCache(enabled=True):
    return _opt(inversion_cache=1 if enabled else 0)


def WithGPU(device=0):
    """Select the CUDA device (the GPU counterpart of the CPU tuning options)."""
    return _opt(device=int(device))


def _noop(*_a, **_k):
    return lambda o: None


# CPU scheduling / ISA options of the reference: accepted, no effect on a GPU.
WithMaxGoroutines = WithAutoGoroutines = WithMinSplitSize = _noop
WithSSSE3 = WithAVX2 = WithSSE2 = WithAVX512 = WithGFNI = WithAVXGFNI = _noop
WithConcurrentStreams = WithConcurrentStreamReads = WithConcurrentStreamWrites = _noop
WithWorkAllocator = _noop


def WithStreamBlockSize(n):
    """Per-shard block size of a StreamEncoder round (options.go:159-167)."""
    return _opt(stream_block=int(n))


# ---- device contexts ----------------------------------------------------------
class Context:
    """One librsgpu context (stream + scratch) per CUDA device, kept for the
    life of the process (like the reference's package-level tables)."""
    _by_device = {}

    def __init__(self, device):
        self.device = device
        h = ctypes.c_void_p()
        check(L.lib().rsgpu_ctx_create(device, ctypes.byref(h)))
        self.handle = h

    @classmethod
    def get(cls, device=0):
        if device not in cls._by_device:
            cls._by_device[device] = cls(device)
        return cls._by_device[device]

    def bind_current_stream(self):
        """Run library work on torch's current stream, ordered with torch ops."""
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(L.lib().rsgpu_ctx_set_stream(self.handle, ctypes.c_void_p(s)))


class _DeviceBlock:
    """One device allocation of rsgpu_alloc_shards, freed with rsgpu_free."""

    def __init__(self, ctx, ptr):
        self.ctx, self.ptr = ctx, ptr

    def __del__(self):
        try:
            L.lib().rsgpu_free(self.ctx.handle, ctypes.c_void_p(self.ptr))
        except Exception:
            pass


class _ShardView:
    """A shard of a _DeviceBlock exposed through __cuda_array_interface__ (the
    tensor made from it keeps this object, and so the block, alive)."""

    def __init__(self, block, ptr, n):
        self._block = block
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _is_device(t):
    return isinstance(t, torch.Tensor) and t.is_cuda


def _size(shards):
    for s in shards:
        if s is not None and len(s):
            return len(s)
    return 0


def _ptr(t):
    if t is None or len(t) == 0:
        return None
    if isinstance(t, np.ndarray):
        if not t.flags["C_CONTIGUOUS"] or t.dtype != np.uint8:
            raise ErrInvalidInput("shards must be contiguous uint8")
        return t.ctypes.data
    if t.dtype != torch.uint8 or not t.is_contiguous():
        raise ErrInvalidInput("shards must be contiguous uint8")
    return t.data_ptr()


class Encoder:
    """Encoder + Extensions (reedsolomon.go:25-165) over librsgpu."""

    def __init__(self, data_shards, parity_shards, opts):
        o = {"device": 0, "matrix": "default", "fast_one_parity": 0, "leopard": 0,
             "inversion_cache": 1, "custom": None, "host_only": False, "stream_block": 0}
        for f in opts:
            f(o)
        self._o = o
        lib = L.lib()
        ro = L.RsOptions()
        lib.rsgpu_options_init(ctypes.byref(ro))
        ro.matrix_kind = _MATRIX[o["matrix"]]
        ro.fast_one_parity = o["fast_one_parity"]
        ro.leopard = o["leopard"]
        ro.inversion_cache = o["inversion_cache"]
        self._custom = None
        if o["custom"] is not None:
            self._custom = np.ascontiguousarray(o["custom"])
            ro.custom_matrix = self._custom.ctypes.data
            ro.custom_rows, ro.custom_cols = self._custom.shape
        self.ctx = None if o["host_only"] else Context.get(o["device"])
        h = ctypes.c_void_p()
        check(lib.rsgpu_encoder_new(self.ctx.handle if self.ctx else None, data_shards, parity_shards,
                                    ctypes.byref(ro), ctypes.byref(h)))
        self._h = h
        k, p, mult, codec = (ctypes.c_int() for _ in range(4))
        check(lib.rsgpu_encoder_info(h, ctypes.byref(k), ctypes.byref(p), ctypes.byref(mult), ctypes.byref(codec)))
        self._k, self._p, self._mult, self.codec = k.value, p.value, mult.value, codec.value

    def __del__(self):
        try:
            L.lib().rsgpu_encoder_free(self._h)
        except Exception:
            pass

    def PrepareKernels(self):
        """Compiles now the generated kernels this encoder's Encode and Verify
        use (no device needed); returns how many are ready."""
        n = L.lib().rsgpu_encoder_prepare_kernels(self._h)
        if n < 0:
            check(n)
        return n

    # Extensions
    def DataShards(self):
        return self._k

    def ParityShards(self):
        return self._p

    def TotalShards(self):
        return self._k + self._p

    def ShardSizeMultiple(self):
        return self._mult

    def Matrix(self):
        m = np.zeros((self.TotalShards(), self._k), dtype=np.uint8)
        check(L.lib().rsgpu_encoder_matrix(self._h, m.ctypes.data))
        return m

    def AllocAligned(self, each):
        """AllocAligned (unsafe.go:19-43): TotalShards device shards of `each`
        bytes carved from one allocation made by rsgpu_alloc_shards, each
        starting on a 64-byte boundary.  The shards are uint8 CUDA tensors;
        the allocation is freed when the last of them is released."""
        if self.ctx is None:
            raise ErrNoDevice("encoder has no device context")
        n = self.TotalShards()
        ptrs = (ctypes.c_void_p * n)()
        check(L.lib().rsgpu_alloc_shards(self.ctx.handle, n, int(each), ptrs))
        block = _DeviceBlock(self.ctx, ptrs[0])
        dev = torch.device("cuda", self.ctx.device)
        return [torch.as_tensor(_ShardView(block, ptrs[i], each), device=dev) for i in range(n)]

    # --- helpers
    def _prep(self, shards, nilok):
        if len(shards) != self.TotalShards():
            raise ErrTooFewShards("too few shards given")
        size = _size(shards)
        if size == 0:
            raise ErrShardNoData("no shard data")
        for s in shards:
            n = 0 if s is None else len(s)
            if n != size and (n != 0 or not nilok):
                raise ErrShardSize("shard sizes do not match")
        dev = any(_is_device(s) for s in shards if s is not None and len(s))
        return size, dev

    def _bind(self):
        if self.ctx is None:
            raise ErrNoDevice("encoder has no device context")
        self.ctx.bind_current_stream()

    # Encoder
    def Encode(self, shards):
        size, dev = self._prep(shards, nilok=False)
        lib = L.lib()
        arr = L.ptr_array([_ptr(s) for s in shards])
        if dev:
            self._bind()
            check(lib.rsgpu_encode(self._h, arr, size))
        else:
            check(lib.rsgpu_encode_host(self._h, arr, size))

    def EncodeIdx(self, data_shard, idx, parity):
        if len(parity) != self._p:
            raise ErrTooFewShards("too few shards given")
        if self._p == 0:
            return
        if idx < 0 or idx >= self._k:
            raise ErrInvShardNum("invalid shard index")
        size = _size(parity)
        if size == 0:
            raise ErrShardNoData("no shard data")
        if any(p is None or len(p) != size for p in parity) or len(data_shard) != size:
            raise ErrShardSize("shard sizes do not match")
        if self._on_device([data_shard] + list(parity)):
            self._bind()
            check(L.lib().rsgpu_encode_idx(self._h, _ptr(data_shard), idx,
                                           L.ptr_array([_ptr(p) for p in parity]), size))
        else:
            check(L.lib().rsgpu_encode_idx_host(self._h, _ptr(data_shard), idx,
                                                L.ptr_array([_ptr(p) for p in parity]), size))

    def Update(self, shards, newDatashards):
        """Update (reedsolomon.go:762-853): parity += P * (old ^ new) for every
        data shard with new data; the old data shard is left holding old ^ new,
        as in the reference.  Shards all on the device or all in host memory."""
        if self.codec != RS_CODEC_CLASSIC:
            raise ErrNotSupported("operation not supported")
        if len(shards) != self.TotalShards() or len(newDatashards) != self._k:
            raise ErrTooFewShards("too few shards given")
        size, dev = self._prep(shards, nilok=True)
        nsize = _size(newDatashards)
        if nsize == 0:
            raise ErrShardNoData("no shard data")
        for s in newDatashards:
            n = 0 if s is None else len(s)
            if n != nsize and n != 0:
                raise ErrShardSize("shard sizes do not match")
        for i, s in enumerate(newDatashards):
            if s is not None and len(s) and (shards[i] is None or not len(shards[i])):
                raise ErrInvalidInput("invalid input")
        if any(p is None or not len(p) for p in shards[self._k:]):
            raise ErrInvalidInput("invalid input")
        if nsize != size:  # the reference would index past the shorter slices
            raise ErrShardSize("shard sizes do not match")
        new = [s if (s is not None and len(s)) else None for s in newDatashards]
        live = [s for s in list(shards) + new if s is not None and len(s)]
        if self._on_device(live):
            self._bind()
            check(L.lib().rsgpu_update(self._h, L.ptr_array([_ptr(s) for s in shards]),
                                       L.ptr_array([_ptr(s) for s in new]), size))
        else:
            check(L.lib().rsgpu_update_host(self._h, L.ptr_array([_ptr(s) for s in shards]),
                                            L.ptr_array([_ptr(s) for s in new]), size))

    def DecodeIdx(self, dst, expectInput, input):
        """DecodeIdx (reedsolomon.go:1464-1617): accumulate this call's inputs
        into the non-None dst shards (zeroed by the caller before the first
        call); expectInput=None merges two partial results (dst ^= input)."""
        if self.codec != RS_CODEC_CLASSIC:
            raise ErrNotSupported("operation not supported")
        lib = L.lib()
        if expectInput is None:
            if len(dst) != len(input):
                raise ErrInvalidInput("dst and input must have same length for merging")
            for i, x in enumerate(input):
                if x is not None:
                    if dst[i] is None:
                        raise ErrInvalidInput("input[%d] provided but dst[%d] is nil" % (i, i))
                    if len(dst[i]) != len(x):
                        raise ErrInvalidShardSize("dst[%d] size != input[%d] size" % (i, i))
            pad = [None] * (self.TotalShards() - 1)
            for i, x in enumerate(input):  # pairs may differ in size: one merge call per pair
                if x is not None and len(x):
                    if self._on_device([x, dst[i]]):
                        self._bind()
                        f = lib.rsgpu_decode_idx
                    else:
                        f = lib.rsgpu_decode_idx_host
                    check(f(self._h, L.ptr_array([_ptr(dst[i])] + pad), None, L.ptr_array([_ptr(x)] + pad), len(x)))
            return
        n = self.TotalShards()
        if len(expectInput) != n or len(dst) != n or len(input) != n:
            raise ErrInvalidInput("expectInput, dst and input must have totalShards entries")
        for i in range(n):
            if input[i] is not None and not expectInput[i]:
                raise ErrInvalidInput("unexpected input at index %d" % i)
            if expectInput[i] and dst[i] is not None:
                raise ErrInvalidInput("dst[%d] should be nil" % i)
        if sum(1 for e in expectInput if e) < self._k:
            raise ErrTooFewShards("too few shards given")
        size = 0
        for x in input:
            if x is not None:
                if size == 0:
                    size = len(x)
                elif len(x) != size:
                    raise ErrInvalidShardSize("input sizes differ")
        for d in dst:
            if d is not None and len(d) != size:
                raise ErrInvalidShardSize("dst size differs from the input size")
        live = [x for x in list(dst) + list(input) if x is not None and len(x)]
        if not live:
            return
        if self._on_device(live):
            self._bind()
            f = lib.rsgpu_decode_idx
        else:
            f = lib.rsgpu_decode_idx_host
        check(f(self._h, L.ptr_array([_ptr(d) for d in dst]), L.u8_array([1 if e else 0 for e in expectInput]),
                L.ptr_array([_ptr(x) for x in input]), size))

    @staticmethod
    def _on_device(tensors):
        """True when every tensor is on the device, False when every one is in
        host memory (the *_host entry points move the bytes); mixed sets are
        refused."""
        dev = [_is_device(t) for t in tensors]
        if all(dev):
            return True
        if not any(dev):
            return False
        raise ErrNotSupported("shards must be all on the device or all in host memory")

    def Split(self, data):
        """Split (reedsolomon.go:1803-1856; leopard.go:320-370) of a 1-D uint8
        CUDA tensor into k+p shards of ceil(len/k) bytes (Leopard: rounded up
        to 64).  Full shards are views of `data`; the rest share one zeroed
        padding buffer."""
        return self.SplitCap(data, len(data), len(data))

    def SplitCap(self, buf, length, cap):
        """Split of buf[:length] with buf[length:cap] usable as spare capacity,
        as the reference uses a slice's capacity (those bytes are zeroed)."""
        if not _is_device(buf) or buf.dtype != torch.uint8 or not buf.is_contiguous():
            raise ErrNotSupported("Split takes a contiguous uint8 device tensor")
        cap = max(int(cap), int(length))
        if cap > buf.numel():
            raise ErrInvalidInput("cap exceeds the buffer")
        lib = L.lib()
        per, pad = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib.rsgpu_split_plan(self._h, int(length), cap, ctypes.byref(per), ctypes.byref(pad)))
        padding = torch.empty(pad.value + 64, dtype=torch.uint8, device=buf.device) if pad.value else None
        pad_off = 0
        if padding is not None:
            pad_off = (-padding.data_ptr()) % 64
        ptrs = L.ptr_array([None] * self.TotalShards())
        self._bind()
        check(lib.rsgpu_split(self._h, _ptr(buf) if length else None, int(length), cap,
                              None if padding is None else ctypes.c_void_p(padding.data_ptr() + pad_off),
                              pad.value, ptrs, ctypes.byref(per)))
        out = []
        base, pbase = buf.data_ptr(), (padding.data_ptr() + pad_off) if padding is not None else None
        for i in range(self.TotalShards()):
            addr = ptrs[i]
            if base <= addr < base + cap:
                out.append(buf[addr - base:addr - base + per.value])
            else:
                off = addr - pbase
                out.append(padding[pad_off + off:pad_off + off + per.value])
        return out

    def Join(self, dst, shards, outSize):
        """Join (reedsolomon.go:1858-1898): the first outSize bytes of the data
        shards into `dst` (a uint8 tensor, device or host, of >= outSize bytes,
        or an object with write())."""
        if len(shards) < self._k:
            raise ErrTooFewShards("too few shards given")
        have = 0
        for s in shards[:self._k]:
            if s is None:
                raise ErrReconstructRequired("reconstruction required")
            have += len(s)
            if have >= outSize:
                break
        if have < outSize:
            raise ErrShortData("not enough data to fill the number of requested shards")
        sizes = {len(s) for s in shards[:self._k] if s is not None}
        if len(sizes) > 1:
            raise ErrShardSize("shard sizes do not match")
        size = sizes.pop()
        lib = L.lib()
        data = [s if (s is not None) else None for s in shards[:self._k]] + [None] * self._p
        if isinstance(dst, torch.Tensor):
            if dst.numel() < outSize or dst.dtype != torch.uint8 or not dst.is_contiguous():
                raise ErrShortData("dst is shorter than outSize")
            self._bind()
            check(lib.rsgpu_join(self._h, ctypes.c_void_p(dst.data_ptr()), L.ptr_array([_ptr(s) for s in data]),
                                 size, int(outSize)))
            return
        out = torch.empty(int(outSize), dtype=torch.uint8, pin_memory=True)
        self._bind()
        check(lib.rsgpu_join(self._h, ctypes.c_void_p(out.data_ptr()), L.ptr_array([_ptr(s) for s in data]),
                             size, int(outSize)))
        dst.write(out.numpy().tobytes())

    def Verify(self, shards):
        size, dev = self._prep(shards, nilok=False)
        ok = ctypes.c_int()
        if self._on_device(shards):
            self._bind()
            check(L.lib().rsgpu_verify(self._h, L.ptr_array([_ptr(s) for s in shards]), size, ctypes.byref(ok)))
        else:
            check(L.lib().rsgpu_verify_host(self._h, L.ptr_array([_ptr(s) for s in shards]), size,
                                            ctypes.byref(ok)))
        return bool(ok.value)

    def _reconstruct(self, shards, data_only, required=None):
        if len(shards) != self.TotalShards():
            raise ErrTooFewShards("too few shards given")
        size, dev = self._prep(shards, nilok=True)
        present = [1 if (s is not None and len(s)) else 0 for s in shards]
        n = self.TotalShards()
        if self.codec != RS_CODEC_CLASSIC:
            # leopard.go:378-391: all missing data shards are recovered; parity
            # too for Reconstruct, or ReconstructSome with a full-length required.
            recover_all = (not data_only) if required is None else len(required) == n
            want = [not present[i] and (i < self._k or recover_all) for i in range(n)]
        elif required is not None:
            req = [bool(r) for r in required]
            want = [not present[i] and i < len(req) and req[i] for i in range(n)]
        else:
            want = [not present[i] and (i < self._k or not data_only) for i in range(n)]
        if not dev:
            return self._reconstruct_host(shards, present, want, size, data_only, required)
        self._bind()
        device = self.ctx.device
        outs = list(shards)
        for i in range(n):
            if want[i]:
                outs[i] = torch.empty(size, dtype=torch.uint8, device="cuda:%d" % device)
        ptrs = L.ptr_array([_ptr(s) for s in outs])
        pres = L.u8_array(present)
        written = (ctypes.c_uint8 * n)()
        lib = L.lib()
        if required is not None:
            reqa = L.u8_array([1 if r else 0 for r in required])
            check(lib.rsgpu_reconstruct_some(self._h, ptrs, pres, reqa, len(required), size, written))
        elif data_only:
            check(lib.rsgpu_reconstruct_data(self._h, ptrs, pres, size, written))
        else:
            check(lib.rsgpu_reconstruct(self._h, ptrs, pres, size, written))
        for i in range(n):
            if written[i]:
                shards[i] = outs[i]

    def Reconstruct(self, shards):
        self._reconstruct(shards, data_only=False)

    def ReconstructData(self, shards):
        self._reconstruct(shards, data_only=True)

    def ReconstructSome(self, shards, required):
        if len(required) not in (self._k, self.TotalShards()):
            raise ErrInvalidInput("invalid input")
        self._reconstruct(shards, data_only=len(required) == self._k, required=required)

    def _reconstruct_host(self, shards, present, want, size, data_only, required):
        """Host buffers: missing outputs are allocated as pinned CPU tensors, PCIe copies run inside."""
        n = self.TotalShards()
        outs = list(shards)
        for i in range(n):
            if want[i]:
                outs[i] = torch.empty(size, dtype=torch.uint8, pin_memory=True)
        written = (ctypes.c_uint8 * n)()
        ptrs = L.ptr_array([_ptr(s) for s in outs])
        if required is not None:
            check(L.lib().rsgpu_reconstruct_some_host(self._h, ptrs, L.u8_array(present),
                                                      L.u8_array([1 if r else 0 for r in required]),
                                                      len(required), size, written))
        else:
            check(L.lib().rsgpu_reconstruct_host(self._h, ptrs, L.u8_array(present), size, int(data_only), written))
        for i in range(n):
            if written[i]:
                shards[i] = outs[i]

    def DecodePlan(self, present, data_only=False, required=None):
        """The decode rows, output and input indices reconstruct would use (host only)."""
        n, k = self.TotalShards(), self._k
        rows = np.zeros((n, k), dtype=np.uint8)
        out_idx = (ctypes.c_int * n)()
        in_idx = (ctypes.c_int * k)()
        n_out = ctypes.c_int()
        req = L.u8_array(required) if required is not None else None
        check(L.lib().rsgpu_decode_plan(self._h, L.u8_array(present), int(data_only), req,
                                        len(required) if required is not None else 0,
                                        rows.ctypes.data, out_idx, ctypes.byref(n_out), in_idx))
        no = n_out.value
        return rows[:no].copy(), list(out_idx[:no]), (list(in_idx[:k]) if no else [])


def New(data_shards, parity_shards, *opts):
    """reedsolomon.New (reedsolomon.go:425)."""
    return Encoder(data_shards, parity_shards, opts)


# ---- StreamEncoder (streaming.go) --------------------------------------------
class StreamReadError(RSError):
    """A reader failed (streaming.go:93-109); .stream is its shard index."""
    code = -14

    def __init__(self, err, stream):
        super().__init__("error reading stream %d: %s" % (stream, err))
        self.err, self.stream = err, stream


class StreamWriteError(RSError):
    """A writer failed (streaming.go:111-127); .stream is its shard index."""
    code = -15

    def __init__(self, err, stream):
        super().__init__("error writing stream %d: %s" % (stream, err))
        self.err, self.stream = err, stream




class _StreamIO:
    """ctypes callbacks over Python readers (read/readinto) and writers (write)."""

    def __init__(self, readers, writers):
        self.readers, self.writers = readers, writers
        self.exc = None
        self.read_fn = L.READ_FN(self._read)
        self.write_fn = L.WRITE_FN(self._write)

    def _read(self, _user, shard, buf, n):
        try:
            r = self.readers[shard]
            view = (ctypes.c_ubyte * n).from_address(buf)
            if hasattr(r, "readinto"):
                got = r.readinto(memoryview(view).cast("B"))
                return int(got or 0)
            data = r.read(n)
            ctypes.memmove(buf, data, len(data))
            return len(data)
        except Exception as e:  # reported as StreamReadError
            self.exc = e
            return -1

    def _write(self, _user, shard, buf, n):
        try:
            w = self.writers[shard]
            m = w.write(ctypes.string_at(buf, n))
            if m is not None and m != n:
                raise IOError("short write")
            return 0
        except Exception as e:
            self.exc = e
            return 1

    def check(self, rc, shard):
        if rc == -14:
            raise StreamReadError(self.exc, shard)
        if rc == -15:
            raise StreamWriteError(self.exc, shard)
        check(rc)


class StreamEncoder:
    """StreamEncoder (streaming.go:23-91) over librsgpu: shards are file-like
    objects, processed in blocks (WithStreamBlockSize, default 4 MiB)."""

    def __init__(self, enc, block):
        self.enc, self.block = enc, block

    def _run(self, readers, writers, fn):
        io = _StreamIO(readers, writers)
        shard = ctypes.c_int(-1)
        self.enc._bind()
        rc = fn(io, shard)
        io.check(rc, shard.value)

    def Encode(self, data, parity):
        k, p = self.enc.DataShards(), self.enc.ParityShards()
        if len(data) != k or len(parity) != p:
            raise ErrTooFewShards("too few shards given")
        readers = list(data) + [None] * p
        writers = [None] * k + list(parity)
        self._run(readers, writers, lambda io, sh: L.lib().rsgpu_stream_encode(
            self.enc._h, io.read_fn, io.write_fn, None, self.block, ctypes.byref(sh)))

    def Verify(self, shards):
        if len(shards) != self.enc.TotalShards():
            raise ErrTooFewShards("too few shards given")
        ok = ctypes.c_int()
        self._run(list(shards), [], lambda io, sh: L.lib().rsgpu_stream_verify(
            self.enc._h, io.read_fn, None, self.block, ctypes.byref(ok), ctypes.byref(sh)))
        return bool(ok.value)

    def Reconstruct(self, valid, fill):
        n = self.enc.TotalShards()
        if len(valid) != n or len(fill) != n:
            raise ErrTooFewShards("too few shards given")
        v = L.u8_array([0 if r is None else 1 for r in valid])
        f = L.u8_array([0 if w is None else 1 for w in fill])
        self._run(list(valid), list(fill), lambda io, sh: L.lib().rsgpu_stream_reconstruct(
            self.enc._h, v, f, io.read_fn, io.write_fn, None, self.block, ctypes.byref(sh)))

    def Split(self, data, dst, size):
        """streaming.go:569-603: `size` bytes of `data` into k writers, zero padded."""
        if size == 0:
            raise ErrShortData("not enough data to fill the number of requested shards")
        k = self.enc.DataShards()
        if len(dst) != k:
            raise ErrInvShardNum("cannot create Encoder with less than one data shard or less than zero parity shards")
        for i, w in enumerate(dst):
            if w is None:
                raise StreamWriteError(ErrShardNoData("no shard data"), i)
        per = (size + k - 1) // k
        left = size
        for i in range(k):
            want = min(per, left)
            got = b""
            while len(got) < want:
                chunk = data.read(want - len(got))
                if not chunk:
                    break
                got += chunk
            if len(got) != want:
                raise ErrShortData("not enough data to fill the number of requested shards")
            left -= want
            dst[i].write(got + bytes(per - want))

    def Join(self, dst, shards, outSize):
        """streaming.go:515-553: the first outSize bytes of the data shard readers."""
        k = self.enc.DataShards()
        if len(shards) < k:
            raise ErrTooFewShards("too few shards given")
        for i in range(k):
            if shards[i] is None:
                raise StreamReadError(ErrShardNoData("no shard data"), i)
        left = outSize
        for i in range(k):
            while left:
                chunk = shards[i].read(min(left, 1 << 20))
                if not chunk:
                    break
                dst.write(chunk)
                left -= len(chunk)
        if left:
            raise ErrShortData("not enough data to fill the number of requested shards")


def NewStream(data_shards, parity_shards, *opts):
    """reedsolomon.NewStream (streaming.go:146-185): at most 256 shards."""
    if data_shards + parity_shards > 256:
        raise ErrMaxShardNum("cannot create Encoder with more than 256 data+parity shards")
    enc = Encoder(data_shards, parity_shards, opts)
    if enc.codec != RS_CODEC_CLASSIC:
        raise ErrNotSupported("operation not supported")
    return StreamEncoder(enc, enc._o["stream_block"] or (4 << 20))


def HostOnly():
    """Option: build the encoder without a device context (planning only)."""
    return _opt(host_only=True)


# ---- kernel seam (LowLevel / codeSomeShards) ---------------------------------
def code_some_shards(rows, inputs, outputs, clear=True, start=0, stop=None, device=0):
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    n_out, n_in = rows.shape
    ctx = Context.get(device)
    ctx.bind_current_stream()
    stop = len(inputs[0]) if stop is None else stop
    check(L.lib().rsgpu_code_some_shards(ctx.handle, rows.ctypes.data, n_in, n_out,
                                         L.ptr_array([t.data_ptr() for t in inputs]),
                                         L.ptr_array([t.data_ptr() for t in outputs]),
                                         start, stop, int(bool(clear))))


def check_some_shards(rows, inputs, to_check, device=0):
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    n_out, n_in = rows.shape
    ctx = Context.get(device)
    ctx.bind_current_stream()
    ok = ctypes.c_int()
    check(L.lib().rsgpu_check_some_shards(ctx.handle, rows.ctypes.data, n_in, n_out,
                                          L.ptr_array([t.data_ptr() for t in inputs]),
                                          L.ptr_array([t.data_ptr() for t in to_check]),
                                          len(inputs[0]), ctypes.byref(ok)))
    return bool(ok.value)


def gal_mul_slice(c, inp, out, xor=False, device=0):
    ctx = Context.get(device)
    ctx.bind_current_stream()
    check(L.lib().rsgpu_gal_mul_slice(ctx.handle, int(c), inp.data_ptr(), out.data_ptr(), len(inp), int(xor)))


def slice_xor(inp, out, device=0):
    ctx = Context.get(device)
    ctx.bind_current_stream()
    check(L.lib().rsgpu_slice_xor(ctx.handle, inp.data_ptr(), out.data_ptr(), len(inp)))


def build_matrix(kind, data_shards, total_shards):
    out = np.zeros((total_shards, data_shards), dtype=np.uint8)
    check(L.lib().rsgpu_build_matrix(_MATRIX[kind], data_shards, total_shards, out.ctypes.data))
    return out


def invert_matrix(m):
    m = np.ascontiguousarray(m, dtype=np.uint8)
    out = np.zeros_like(m)
    check(L.lib().rsgpu_invert_matrix(m.ctypes.data, m.shape[0], out.ctypes.data))
    return out


# ---- GF(2^8) kernel variants and tuning ---------------------------------------
MODES = {"write": 0, "xor": 1, "verify": 2}
VARIANT_XORNET = 7  # the bit-sliced XOR network generated per coefficient matrix


def autotune(n_in, n_out, shard_bytes, mode="write", reps=3, device=0):
    """Times every GF(2^8) kernel variant for this geometry on scratch data
    and keeps the fastest for its input count, output group, mode and size
    bucket.  Returns (best variant, {variant: ms}); variants that cannot run
    here (no NVRTC for the XOR network) are absent from the dict."""
    lib = L.lib()
    ms = (ctypes.c_float * lib.rsgpu_num_variants())()
    best = ctypes.c_int(-1)
    check(lib.rsgpu_autotune_gf8(Context.get(device).handle, n_in, n_out, shard_bytes, MODES[mode], reps, ms,
                                 ctypes.byref(best)))
    return best.value, {v: x for v, x in enumerate(ms) if x < 1e29}


def record_variant(n_in, n_out, shard_bytes, variant, mode="write"):
    """Installs a saved tuning choice without timing (None removes it)."""
    check(L.lib().rsgpu_record_variant(n_in, n_out, shard_bytes, MODES[mode], -1 if variant is None else variant))


def force_variant(variant):
    """Uses one variant for every launch (None: back to the tuned choice)."""
    check(L.lib().rsgpu_force_variant(-1 if variant is None else variant))


def generated_kernels_available():
    """True when the per-matrix XOR-network kernels can be compiled (NVRTC)."""
    return bool(L.lib().rsgpu_xornet_available())


def wait_generated_kernels():
    """Waits for queued background compiles; returns how many generated
    kernels this process holds."""
    return L.lib().rsgpu_xornet_sync()


# ---- batched mixed-geometry execution ---------------------------------------
RS_JOB_ENCODE, RS_JOB_RECONSTRUCT, RS_JOB_RECONSTRUCT_DATA, RS_JOB_VERIFY = 0, 1, 2, 3
BATCH_MODES = {"persistent": 0, "per_stripe": 1, "graph": 2}


class Batch:
    """Many stripe operations of mixed geometry run as one launch.

    add_* plan on the host (matrices, decode rows); run() executes every
    planned job on the GPU: mode "persistent" (one launch), "per_stripe"
    (one launch per stripe operation) or "graph" (those launches captured
    once into a CUDA graph).  Shards are CUDA uint8 tensors; reconstruct
    outputs must be preallocated tensors, with `present` marking valid shards.
    """

    def __init__(self, device=0, *opts):
        self.ctx = Context.get(device)
        o = {"matrix": "default", "fast_one_parity": 0, "inversion_cache": 1}
        for f in opts:
            f(o)
        ro = L.RsOptions()
        L.lib().rsgpu_options_init(ctypes.byref(ro))
        ro.matrix_kind = _MATRIX[o["matrix"]]
        ro.fast_one_parity = o["fast_one_parity"]
        ro.inversion_cache = o["inversion_cache"]
        h = ctypes.c_void_p()
        check(L.lib().rsgpu_batch_create(self.ctx.handle, ctypes.byref(ro), ctypes.byref(h)))
        self._h = h
        self.n = 0

    def __del__(self):
        try:
            L.lib().rsgpu_batch_destroy(self._h)
        except Exception:
            pass

    def _add(self, op, k, p, shards, present=None):
        ptrs = L.ptr_array([_ptr(s) for s in shards])
        st = L.RsStripe(op, k, p, _size(shards), ctypes.cast(ptrs, ctypes.c_void_p),
                        ctypes.cast(L.u8_array(present), ctypes.c_void_p) if present is not None else None)
        keep = (ptrs, st)
        if present is not None:
            pres = L.u8_array(present)
            st.present = ctypes.cast(pres, ctypes.c_void_p)
            keep = keep + (pres,)
        check(L.lib().rsgpu_batch_add(self._h, ctypes.byref(st), 1))
        self.n += 1
        return self.n - 1

    def add_encode(self, k, p, shards):
        return self._add(RS_JOB_ENCODE, k, p, shards)

    def add_verify(self, k, p, shards):
        return self._add(RS_JOB_VERIFY, k, p, shards)

    def add_reconstruct(self, k, p, shards, present, data_only=False):
        return self._add(RS_JOB_RECONSTRUCT_DATA if data_only else RS_JOB_RECONSTRUCT, k, p, shards, present)

    def set_tile(self, tile_bytes):
        check(L.lib().rsgpu_batch_set_tile(self._h, int(tile_bytes)))

    def autotune(self, reps=2):
        """Times the persistent launch over this batch's jobs for several
        tile sizes and CTAs per SM and keeps the fastest: (tile bytes, CTAs
        per SM, ms per run)."""
        self.ctx.bind_current_stream()
        tile, ctas, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        check(L.lib().rsgpu_batch_autotune(self._h, int(reps), ctypes.byref(tile), ctypes.byref(ctas),
                                           ctypes.byref(ms)))
        return tile.value, ctas.value, ms.value

    def run(self, mode="persistent", wait=True):
        self.ctx.bind_current_stream()
        f = L.lib().rsgpu_batch_run if wait else L.lib().rsgpu_batch_run_async
        check(f(self._h, BATCH_MODES[mode]))

    def results(self):
        ok = (ctypes.c_int * max(1, self.n))()
        check(L.lib().rsgpu_batch_results(self._h, ok, self.n))
        return [bool(ok[i]) for i in range(self.n)]

    def info(self):
        ns, nj = ctypes.c_int(), ctypes.c_int()
        nt, by = ctypes.c_longlong(), ctypes.c_double()
        check(L.lib().rsgpu_batch_info(self._h, ctypes.byref(ns), ctypes.byref(nj), ctypes.byref(nt), ctypes.byref(by)))
        return {"stripes": ns.value, "jobs": nj.value, "tiles": nt.value, "bytes": by.value}


# ---- request server ------------------------------------------------------------
class Server:
    """Continuous-batching request server over device-resident stripes.

    submit() queues a request (op, geometry, CUDA shard tensors); the server
    thread admits requests in arrival order under an in-flight byte budget
    and an HBM arena for reconstruct outputs left as None, and runs them as
    micro-batches on `streams` streams.  poll() returns completions with
    their submit-to-completion latency; outputs(ticket) gives the shard
    device pointers after completion; release(ticket) frees arena outputs.
    """
    OPS = {"encode": RS_JOB_ENCODE, "reconstruct": RS_JOB_RECONSTRUCT,
           "reconstruct_data": RS_JOB_RECONSTRUCT_DATA, "verify": RS_JOB_VERIFY}

    def __init__(self, arena_bytes=1 << 30, inflight_budget=8 << 30, max_batch=256, streams=4, device=0):
        self.ctx = Context.get(device)
        h = ctypes.c_void_p()
        check(L.lib().rsgpu_server_create(self.ctx.handle, int(arena_bytes), int(inflight_budget), int(max_batch),
                                          int(streams), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def _request(self, op, k, p, shards, present=None, leopard=0, tag=0, size=None):
        """`size` (bytes per shard) defaults to the length of the first shard;
        a smaller size codes that prefix of every shard buffer."""
        n = k + p
        ptrs = L.ptr_array([_ptr(s) if s is not None else None for s in shards])
        req = L.RsRequest(self.OPS[op], k, p, int(leopard), int(size) if size is not None else _size(shards),
                          ctypes.cast(ptrs, ctypes.c_void_p), None, int(tag), 0)
        keep = [ptrs, shards]
        if present is not None:
            pres = L.u8_array(present)
            req.present = ctypes.cast(pres, ctypes.c_void_p)
            keep.append(pres)
        assert len(shards) == n
        return req, keep

    def submit(self, op, k, p, shards, present=None, leopard=0, tag=0, size=None):
        req, keep = self._request(op, k, p, shards, present, leopard, tag, size)
        t = ctypes.c_uint64()
        check(L.lib().rsgpu_server_submit(self._h, ctypes.byref(req), ctypes.byref(t)))
        self._keep[t.value] = (req, keep)
        return t.value

    def replay(self, requests, arrivals_us):
        """requests: list of dicts (op, k, p, shards, present, leopard, tag, size); open-loop arrivals."""
        n = len(requests)
        arr = (L.RsRequest * n)()
        keeps = []
        for i, r in enumerate(requests):
            req, keep = self._request(r["op"], r["k"], r["p"], r["shards"], r.get("present"),
                                      r.get("leopard", 0), r.get("tag", i), r.get("size"))
            arr[i] = req
            keeps.append(keep)
        times = (ctypes.c_double * n)(*[float(x) for x in arrivals_us])
        tickets = (ctypes.c_uint64 * n)()
        check(L.lib().rsgpu_server_replay(self._h, arr, times, n, tickets))
        for i in range(n):
            self._keep[tickets[i]] = (arr, keeps[i], i)
        return list(tickets)

    def _req_of(self, ticket):
        v = self._keep[ticket]
        return v[0][v[2]] if len(v) == 3 else v[0]

    def outputs(self, ticket):
        """Device pointers of the request's shards (reconstructed ones included)."""
        req = self._req_of(ticket)
        n = req.data_shards + req.parity_shards
        arr = ctypes.cast(req.shards, ctypes.POINTER(ctypes.c_void_p))
        return [arr[i] for i in range(n)]

    def verify_result(self, ticket):
        return bool(self._req_of(ticket).result)

    def poll(self, max_n=4096):
        buf = (L.RsCompletion * max_n)()
        n = L.lib().rsgpu_server_poll(self._h, buf, max_n)
        if n < 0:
            check(n)
        return [(buf[i].ticket, buf[i].tag, buf[i].status, buf[i].latency_us) for i in range(n)]

    def poll_detailed(self, max_n=4096):
        """Like poll(), with the admission wait: (ticket, tag, status, latency_us, queue_us)."""
        buf = (L.RsCompletion * max_n)()
        n = L.lib().rsgpu_server_poll(self._h, buf, max_n)
        if n < 0:
            check(n)
        return [(buf[i].ticket, buf[i].tag, buf[i].status, buf[i].latency_us, buf[i].queue_us) for i in range(n)]

    def wait_idle(self, timeout_ms=60000):
        check(L.lib().rsgpu_server_wait_idle(self._h, int(timeout_ms)))

    def release(self, ticket):
        check(L.lib().rsgpu_server_release(self._h, int(ticket)))
        self._keep.pop(ticket, None)

    def stats(self):
        st = L.RsServerStats()
        check(L.lib().rsgpu_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in L.RsServerStats._fields_}

    def reset_stats(self):
        check(L.lib().rsgpu_server_reset_stats(self._h))

    def close(self):
        if self._h:
            L.lib().rsgpu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def memcpy(dst_ptr, src_ptr, nbytes):
    check(L.lib().rsgpu_memcpy(ctypes.c_void_p(dst_ptr), ctypes.c_void_p(src_ptr), int(nbytes)))
