"""Pass schedule of the learned guide (no counterpart in RTLib; modelled on
RTSTreeControllerT's doubling passes, OPX7UtilsPathGuiding.h:1808-1887).

Pass k renders 2^k samples per pixel (the last pass takes the rest of the budget, as the
SD-tree controller does when the remainder is under twice the pass or the ratio of the budget is
spent).  Pass 0 samples the BSDF only and records; every later pass samples the mixture with
probability `fraction` (BUILD).  After every recording pass the network takes `epochs` Adam
passes over the records of that pass; the final pass neither records nor trains.  The records
of a pass are subsampled to the buffer's capacity with a keep probability estimated from the
previous pass.  A time budget ends the schedule early: the pass that crosses 'ratio * budget'
becomes the final one and runs until the budget is spent, one sample per launch."""
from __future__ import annotations

import time

from .tracer import FLAG_BUILD, FLAG_FINAL


def render_learned(tracer, mlp, budget_spp=None, time_budget_s=None, base_flags=1, fraction=0.5, ratio=0.5,
                   epochs=32, batch=4096, sync=None, log=None):
    """Returns the number of samples rendered.  Either budget_spp or time_budget_s (seconds,
    wall clock with a device synchronisation per pass) must be given."""
    import torch
    sync = sync or torch.cuda.synchronize
    t0 = time.perf_counter()
    done, it, keep = 0, 0, 1.0
    npath = tracer.width * tracer.height
    while True:
        elapsed = time.perf_counter() - t0
        if budget_spp is not None:
            remain = budget_spp - done
            if remain <= 0:
                break
            spp = min(remain, 1 << it)
            final = remain - spp < 2 * spp or done >= ratio * budget_spp
            if final:
                spp = remain
        else:
            if elapsed >= time_budget_s:
                break
            spp = 1 << it
            final = elapsed >= ratio * time_budget_s
        flags = (base_flags & 3) | (FLAG_BUILD if it > 0 else 0)
        if final:
            flags |= FLAG_BUILD | FLAG_FINAL
            if budget_spp is not None:
                tracer.render_mlp(spp, flags, mlp, fraction)
                done += spp
            else:
                while time.perf_counter() - t0 < time_budget_s:
                    tracer.render_mlp(1, flags, mlp, fraction)
                    sync()
                    done += 1
            break
        mlp.records(clear=True)
        tracer.render_mlp(spp, flags, mlp, fraction, keep)
        n = mlp.records()
        done += spp
        if n > 0:
            loss = mlp.train(batch=batch, epochs=epochs)
            if log is not None:
                log.append({"pass": it, "spp": spp, "records": min(n, mlp.capacity), "loss": loss})
            per_spp = (n / max(keep, 1e-6)) / spp
            keep = min(1.0, mlp.capacity / max(1.0, per_spp * (1 << (it + 1))))
        sync()
        it += 1
    return done


def render_learned_with_fallback(tracer, mlp, tree, budget_spp=None, time_budget_s=None, base_flags=1, fraction=0.5,
                                 mlp_share=0.5, ratio=0.5, epochs=32, batch=4096, sync=None, log=None):
    """The learned guide with the SD-tree as its fallback: RTSTreeControllerT's pass schedule
    (one sample per launch; build and refine of the tree between passes as in plain SD-tree
    guiding), every launch guided by q = mlp_share * network + (1 - mlp_share) * SD-tree with
    both learning from the same trace vertices, and the network trained after every recording
    pass.  With a time budget the controller's sample budget is unbounded and the launches stop
    when the time is spent.  Returns the number of samples rendered."""
    import torch

    from .sdtree import TRACE_RECORD_AND_SAMPLE, TRACE_SAMPLE, SDTreeController
    from .tracer import FLAG_BUILD, FLAG_FINAL

    sync = sync or torch.cuda.synchronize
    budget = budget_spp if budget_spp is not None else 1 << 30
    ctrl = SDTreeController(tree, budget, iteration_for_built=0, ratio_for_budget=ratio, samples_per_launch=1)
    ctrl.start()
    t0 = time.perf_counter()
    done, keep, last_it, pass_spp = 0, 1.0, 0, 0
    mlp.records(clear=True)
    trained = False
    while True:
        if time_budget_s is not None and time.perf_counter() - t0 >= time_budget_s:
            break
        ctrl.begin()
        st = ctrl.get()
        if not st["executing"]:
            break
        flags = base_flags & 3
        if st["state"] == TRACE_RECORD_AND_SAMPLE:
            flags |= FLAG_BUILD
        elif st["state"] == TRACE_SAMPLE:
            flags |= FLAG_BUILD | FLAG_FINAL
        # before the network has been trained the SD-tree alone guides
        tracer.render_mlp(1, flags, mlp, fraction, keep, fallback=tree, mlp_share=mlp_share if trained else 0.0)
        ctrl.end()
        done += 1
        pass_spp += 1
        st2 = ctrl.get()
        if st2["iteration"] != last_it:  # a pass ended: train on its records
            last_it = st2["iteration"]
            n = mlp.records()
            if n > 0 and not (flags & FLAG_FINAL):
                loss = mlp.train(batch=batch, epochs=epochs)
                trained = True
                if log is not None:
                    log.append({"pass": last_it - 1, "spp": pass_spp, "records": min(n, mlp.capacity), "loss": loss})
                per_spp = (n / max(keep, 1e-6)) / pass_spp
                keep = min(1.0, mlp.capacity / max(1.0, per_spp * 2 * pass_spp))
            mlp.records(clear=True)
            pass_spp = 0
        if time_budget_s is not None:
            sync()
    sync()
    return done
