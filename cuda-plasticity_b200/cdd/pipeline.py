"""Time steps of fields that live in host memory, with the copies overlapped with the computation.

A caller whose states are in (pinned) host memory -- a stream of initial conditions, ensemble
members staged through host RAM, a service that returns each result to the host -- pays one
host-to-device copy and one device-to-host copy per step. Done in order on one stream, a step costs
copy in + compute + copy out. ``HostPipeline`` keeps ``depth`` device buffers and three CUDA
streams (copies in, steps, copies out) ordered by events, so that the copy-in of one step, the step
before it and the copy-out of the one before that run at the same time; PCIe carries both
directions at once. Each step is still one ``Plan.step`` on its own input, and its result reaches
the host buffer given for it. Steps run in the order they are submitted, on the plan's clock.
"""
import torch


class HostPipeline:
    """``step(host_in, host_out)`` queues one step of a 1-instance-or-more plan on the packed field in
    ``host_in`` (pinned, contiguous, plan dtype, ``plan.field_elems`` values) and its copy back to
    ``host_out``; it returns at once. ``synchronize()`` waits for everything queued. A host buffer
    must not be reused before the step that reads or writes it has finished: ``wait(k)`` waits for
    the k-th submitted step."""

    def __init__(self, plan, depth=2):
        self.plan = plan
        self.depth = max(2, int(depth))
        self.bufs = [plan.empty_field() for _ in range(self.depth)]
        self.s_in = torch.cuda.Stream(device=plan.device)
        self.s_run = torch.cuda.Stream(device=plan.device)
        self.s_out = torch.cuda.Stream(device=plan.device)
        self.out_done = [None] * self.depth   # last copy-out from each device buffer
        self.done = []                        # per submitted step: its copy-out event
        self.count = 0

    def _check_host(self, t, name):
        if t.device.type != "cpu" or t.dtype != self.plan.dtype or not t.is_contiguous() \
                or t.numel() != self.plan.field_elems:
            raise ValueError("%s must be a contiguous host tensor of %d %s values"
                             % (name, self.plan.field_elems, self.plan.dtype))

    def step(self, host_in, host_out):
        self._check_host(host_in, "host_in")
        self._check_host(host_out, "host_out")
        i = self.count % self.depth
        b = self.bufs[i]
        with torch.cuda.stream(self.s_in):
            if self.out_done[i] is not None:
                self.s_in.wait_event(self.out_done[i])     # the buffer's previous result has left
            b.copy_(host_in, non_blocking=True)
            ev_in = torch.cuda.Event()
            ev_in.record(self.s_in)
        self.s_run.wait_event(ev_in)
        self.plan.step(b, stream=self.s_run)
        ev_run = torch.cuda.Event()
        ev_run.record(self.s_run)
        with torch.cuda.stream(self.s_out):
            self.s_out.wait_event(ev_run)
            host_out.copy_(b, non_blocking=True)
            ev_out = torch.cuda.Event()
            ev_out.record(self.s_out)
        self.out_done[i] = ev_out
        self.done.append(ev_out)
        self.count += 1
        return ev_out

    def wait(self, k):
        self.done[k].synchronize()

    def synchronize(self):
        for s in (self.s_in, self.s_run, self.s_out):
            s.synchronize()
        self.plan.check_status()
