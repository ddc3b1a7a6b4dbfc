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
                                 mlp_share=0.5, ratio=0.5, epochs=32, batch=4096, sync=None, log=None,
                                 criteria=None):
    """The learned guide with the SD-tree as its fallback: RTSTreeControllerT's pass schedule
    (one sample per launch; build and refine of the tree between passes as in plain SD-tree
    guiding), every launch guided by q = mlp_share * network + (1 - mlp_share) * SD-tree with
    both learning from the same trace vertices, and the network trained after every recording
    pass.  With a time budget the controller's sample budget is unbounded and the launches stop
    when the time is spent.  Returns the number of samples rendered.

    criteria (a list, optional) receives per recording pass, once the network has been trained,
    guide_second_moments of that pass's records, taken after its last launch and before the
    controller builds the SD-tree from them: both guides are judged on records they have not
    been fitted to.  Its cost is inside the time budget."""
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
    # the controller's pass sizes (RTSTreeControllerT::BegTrace), to know a pass's last launch
    remain, pas, per_all, it_m = budget, 0, 0, 0
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
        if pass_spp == 0:
            remain -= pas
            pas = min(remain, 1 << it_m)
            if remain - pas < 2 * pas or per_all >= ratio * budget:
                pas = remain
        tracer.render_mlp(1, flags, mlp, fraction, keep, fallback=tree, mlp_share=mlp_share if trained else 0.0)
        per_all += 1
        if (criteria is not None and trained and pass_spp + 1 == pas and not (flags & FLAG_FINAL)
                and mlp.records() > 0):
            c = guide_second_moments(mlp, tree, fraction, mlp_share)
            if c is not None:
                c["pass"] = it_m
                criteria.append(c)
        ctrl.end()
        done += 1
        pass_spp += 1
        st2 = ctrl.get()
        if st2["iteration"] != last_it:  # a pass ended: train on its records
            last_it = st2["iteration"]
            it_m += 1
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


def _vmf_mixture_pdf(lobes, wi):
    """Density of the 8-lobe mixture (n x 40: mu xyz, kappa, weight per lobe) at wi (n x 3),
    the formula of the tracer's vmf_mixture_pdf."""
    import torch
    L = lobes.view(-1, 8, 5).double()
    mu, k, wgt = L[..., :3], L[..., 3], L[..., 4]
    c = (mu * wi.double()[:, None, :]).sum(-1)
    return (wgt * k / (2 * torch.pi * (1 - torch.exp(-2 * k))) * torch.exp(k * (c - 1))).sum(-1)


def guide_second_moments(mlp, tree, fraction, mlp_share):
    """Per-vertex variance criterion of the guides on the records now in the guide's buffer: for
    a sampling density p, E[f^2 / (q_rec p)] over the records estimates the second moment
    integral of f^2 / p of the one-sample estimator f / p at a vertex (f = w * q_rec, the record's
    luminance of incident radiance times |cos|, q_rec the density it was sampled with).  Returns
    it for the densities the tracer would use with each guide, p = (1 - fraction) cos/pi +
    fraction * q, q the network, the SD-tree, or share * network + (1 - share) * SD-tree, and for
    cosine (BSDF) sampling alone; all surfaces of the scenes it is used on are Lambertian."""
    import torch
    pos, nrm, wo, wi, w, pdf = mlp.record_views()
    n = pos.shape[0]
    if n == 0:
        return None
    lobes = mlp.eval(pos, nrm, wo, raw=False)
    q_net = _vmf_mixture_pdf(lobes, wi)
    q_tree = torch.empty(n, dtype=torch.float32, device=pos.device)
    tree.pdf(pos.contiguous(), wi.contiguous(), q_tree, canonical=False)
    q_tree = q_tree.double()
    bsdf = torch.clamp((nrm.double() * wi.double()).sum(-1), min=0.0) / torch.pi
    f = w.double() * pdf.double()
    ok = (pdf > 0) & (f > 0)

    def moment(p):
        p = p[ok]
        return float((f[ok] ** 2 / (pdf.double()[ok] * p)).mean()) if bool((p > 0).all()) else float("inf")

    mix = lambda q: (1 - fraction) * bsdf + fraction * q
    return {"records": int(ok.sum()), "network": moment(mix(q_net)), "sdtree": moment(mix(q_tree)),
            "mixture": moment(mix(mlp_share * q_net + (1 - mlp_share) * q_tree)), "bsdf": moment(bsdf)}
