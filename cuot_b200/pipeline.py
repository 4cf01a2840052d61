"""Host-facing pipelining of repeated OT-extension steps.

A step takes inputs from pinned host memory, computes on the device and
returns its outputs to pinned host memory.  Run back to back, the device
would idle during each step's device-to-host copy (PCIe-bound: a ferret_b13
step returns 336 MB in ~6.7 ms against ~2.8 ms of compute).  HostPipeline
overlaps that copy with the next step's compute: the outputs are first copied
device-to-device into a staging buffer on the compute stream (HBM speed), and
a separate copy stream moves the staging buffer to the host while the compute
stream runs the next step.  Ordering: the staging copy of step i+1 waits for
the host copy of step i (an event), so at most one step's results are in
flight.

Inputs: with input_sets = 1 they are copied on the compute stream ahead of
the step that reads them, so step i+1's input copy starts only when step i
has finished, at the moment step i's host copy starts.  On B200 the small
input copies then wait behind that large device-to-host copy (sot_n20:
+0.3 ms per 1.8 ms step).  With input_sets = 2 the caller keeps two sets of
device input buffers and gives step j the set `slot` (= j mod 2): its input
copy runs on its own stream as soon as step j-2, the last reader of that
set, has finished, i.e. during step j-1's compute.

Outputs: with per_set_outputs the caller also keeps one set of device output
buffers per input set (step j writes set `slot`); the host copy then reads
them directly, without the device-to-device staging copy, and step j+2 waits
for step j's host copy before it writes that set again.  A step can also
say, per output, when that output is final (`ready`): its host copy then
waits only for that point instead of the whole step, so the outputs that
are final early (a batch's Ferret instances after the LPN, its SOT sizes
largest first) cross PCIe while the rest of the step still computes, and
only the last ones are left after it.
"""
from __future__ import annotations


class HostPipeline:
    def __init__(self, outputs, stream=None, copy_stream=None, input_sets: int = 1,
                 per_set_outputs: bool = False):
        """outputs: the device output tensors, or with per_set_outputs one
        list of them per input set."""
        import torch
        if input_sets not in (1, 2):
            raise ValueError("input_sets must be 1 or 2")
        self.torch = torch
        self.per_set = per_set_outputs
        if per_set_outputs:
            self.outputs = [list(o) for o in outputs]
            if len(self.outputs) != input_sets or len({len(o) for o in self.outputs}) != 1:
                raise ValueError("per_set_outputs needs one equally long output list per input set")
            self.staging = None
        else:
            self.outputs = list(outputs)
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self.copy_stream = copy_stream if copy_stream is not None else torch.cuda.Stream()
        if not per_set_outputs:
            self.staging = [torch.empty_like(o) for o in self.outputs]
        self._d2h_done = None
        self._set_d2h_done = [None] * input_sets  # per output set: its last host copy
        self.input_sets = input_sets
        self.h2d_stream = torch.cuda.Stream() if input_sets > 1 else None
        self._consumed = [None] * input_sets  # per input set: its last reader's compute
        self._count = 0

    @property
    def slot(self) -> int:
        """Input set the next step() must use (0 with input_sets = 1)."""
        return self._count % self.input_sets

    def step(self, inputs, compute, host_outputs, ready=None):
        """inputs: [(host_tensor, device_tensor)] copied host->device first
        (device tensors of input set `slot`); compute(stream) enqueues the
        step's device work; host_outputs: pinned host tensors receiving this
        step's outputs (same shapes as `outputs`).  ready (per_set_outputs
        only): one entry per output, None or a callable ready(copy_stream)
        that makes the copy stream wait until that output is final; the
        outputs are copied in list order, each after the waits of the
        entries up to it, so list them in the order they become final.
        Without it every copy waits for the whole step.  Returns (h2d_bytes,
        d2h_bytes).  Nothing here blocks the host."""
        torch, st = self.torch, self.stream
        if ready is not None:
            if not self.per_set:
                raise ValueError("ready needs per_set_outputs")
            if len(ready) != len(host_outputs) or not ready or ready[0] is None:
                raise ValueError("ready needs one entry per output, the first one a wait")
        h2d = d2h = 0
        slot = self.slot
        cs_in = self.h2d_stream if self.input_sets > 1 else st
        if self.input_sets > 1 and self._consumed[slot] is not None:
            cs_in.wait_event(self._consumed[slot])
        with torch.cuda.stream(cs_in):
            for h, d in inputs:
                d.copy_(h, non_blocking=True)
                h2d += h.numel() * h.element_size()
        if self.input_sets > 1:
            copied = torch.cuda.Event()
            copied.record(cs_in)
            st.wait_event(copied)
        if self.per_set and self._set_d2h_done[slot] is not None:
            st.wait_event(self._set_d2h_done[slot])  # the set's previous results are on the host
        compute(st)
        if self.input_sets > 1:
            done = torch.cuda.Event()
            done.record(st)
            self._consumed[slot] = done
        self._count += 1
        cs = self.copy_stream
        if self.per_set:
            if ready is None:
                done = torch.cuda.Event()
                done.record(st)
                cs.wait_event(done)
            with torch.cuda.stream(cs):
                for j, (o, h) in enumerate(zip(self.outputs[slot], host_outputs)):
                    if ready is not None and ready[j] is not None:
                        ready[j](cs)
                    h.copy_(o, non_blocking=True)
                    d2h += h.numel() * h.element_size()
            self._d2h_done = torch.cuda.Event()
            self._d2h_done.record(cs)
            self._set_d2h_done[slot] = self._d2h_done
            return h2d, d2h
        if self._d2h_done is not None:
            st.wait_event(self._d2h_done)
        with torch.cuda.stream(st):
            for o, s in zip(self.outputs, self.staging):
                s.copy_(o, non_blocking=True)
        staged = torch.cuda.Event()
        staged.record(st)
        cs.wait_event(staged)
        with torch.cuda.stream(cs):
            for s, h in zip(self.staging, host_outputs):
                h.copy_(s, non_blocking=True)
                d2h += h.numel() * h.element_size()
        self._d2h_done = torch.cuda.Event()
        self._d2h_done.record(cs)
        return h2d, d2h

    def join(self):
        """Makes the compute stream wait for the last host copy (so an event
        recorded on it after join() covers every step's results)."""
        if self._d2h_done is not None:
            self.stream.wait_event(self._d2h_done)
