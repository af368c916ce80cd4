"""Workflows and an sprun-compatible runner for the B200 solver.

    python -m seispie_b200.workflow --workdir DIR [--config_file config.ini]

restates scripts/sprun:10-89: config.ini is parsed with configparser, a
``[workflow] inherit = parent`` merges the parent directory's config section
by section (path entries rebased onto the parent, sprun:21-39), paths are
made absolute, and the workflow named by ``[workflow] mode`` loads the
modules it lists, setting ``.config``, ``.path`` and ``.mpi`` on each before
``setup(workflow)`` (sprun:79-86).  Module lookup maps the reference's
sections onto this package: ``[solver] method = b200`` (or ``fd2d``, which
is served by the same plugin) -> seispie_b200.solver.b200, ``[optimize]
method = lbfgs|cg|gd|sgd`` -> seispie_b200.optimize; pre/postprocess are the
reference's empty stubs.  The workflows restate seispie/workflow/*.py.
"""
from __future__ import annotations

import argparse
from configparser import ConfigParser
from os import getcwd, makedirs, path
from time import time


# Sections a child configuration inherits from its parent (the set sprun
# merges, scripts/sprun:24).
INHERITED_SECTIONS = ("workflow", "slurm", "preprocess", "solver", "postprocess", "optimize", "path")


def _adopt(section: str, value: str, parent_rel: str) -> str:
    """A parent's value as the child sees it: entries of [path] are written
    relative to the parent's directory, so they are rebased onto it, except
    'no' (a path switched off); every other value is taken as written."""
    if section == "path" and value != "no":
        return parent_rel + "/" + value
    return value


def merge_configs(child: dict, parent: dict, parent_rel: str) -> dict:
    """child with every key it does not set taken from parent (dicts of
    sections of strings), for the inherited sections only."""
    out = {sec: dict(keys) for sec, keys in child.items()}
    for sec in INHERITED_SECTIONS:
        for key, value in parent.get(sec, {}).items():
            out.setdefault(sec, {}).setdefault(key, _adopt(sec, value, parent_rel))
    return out


def _read(config_path: str) -> dict:
    cp = ConfigParser()
    cp.read(config_path)
    return {sec: dict(cp[sec]) for sec in cp.sections()}


def _resolve(workdir: str, config_file: str) -> dict:
    """The configuration of workdir with its inheritance chain applied."""
    config_path = path.join(workdir, config_file)
    if not path.isdir(workdir) or not path.exists(config_path):
        raise FileNotFoundError(config_path)
    cfg = _read(config_path)
    parent = cfg.get("workflow", {}).get("inherit")
    if parent:
        cfg = merge_configs(cfg, _resolve(path.join(workdir, "..", parent), config_file), "../" + parent)
    return cfg


def parse_config(workdir: str, config_file: str):
    """config.ini of workdir as sprun reads it (scripts/sprun:10-42):
    ``[workflow] inherit = parent`` takes every key the file does not set
    from ../parent/config_file (itself resolved the same way), with the
    parent's paths rebased onto its directory.  Returns (ConfigParser,
    workdir); its sections are what the modules receive as ``.config``."""
    cp = ConfigParser()
    cp.read_dict(_resolve(workdir, config_file))
    return cp, workdir


class _stub:
    """pre/postprocess 'default' (seispie/preprocess/default.py:3-5)."""

    def setup(self, workflow):
        pass


def load_module(section: str, method: str):
    if section == "solver":
        if method not in ("b200", "fd2d"):
            raise ValueError("solver method %r: this package provides the b200 plugin" % method)
        from .solver import b200
        return b200()
    if section == "optimize":
        from . import optimize
        return getattr(optimize, method)()
    if section in ("preprocess", "postprocess"):
        return _stub()
    raise ValueError("unknown section %r" % section)


class forward:
    """workflow/forward.py:4-27."""
    modules = ["solver"]

    def setup(self):
        pass

    def run(self):
        solver = self.solver
        start = time()
        solver.import_model(1)
        solver.import_sources()
        solver.import_stations()
        solver.run_forward()
        print("elapsed time: %.2fs" % (time() - start))


class adjoint:
    """workflow/adjoint.py:5-33."""
    modules = ["solver", "postprocess"]

    def setup(self):
        pass

    def run(self):
        solver = self.solver
        solver.import_model(1)
        solver.import_sources()
        solver.import_stations()
        solver.import_traces()
        start = time()
        solver.import_model(0)
        gradient, _, _ = solver.compute_gradient()
        if not self.mpi or self.mpi.rank() == 0:
            print("")
            print("Elapsed time: %.2fs" % (time() - start))
            solver.export_field(gradient, "kmu")
        self.gradient = gradient


class inversion:
    """workflow/inversion.py:5-27."""
    modules = ["solver", "postprocess", "optimize"]

    def setup(self):
        pass

    def run(self):
        solver = self.solver
        solver.import_model(1)
        solver.import_sources()
        solver.import_stations()
        solver.import_traces()
        solver.import_model(0)
        self.optimize.run()


WORKFLOWS = dict(forward=forward, adjoint=adjoint, inversion=inversion)


def resolve_paths(path_section, workdir: str) -> dict:
    """Absolute paths of the [path] entries that are not switched off."""
    return {key: path.join(workdir, value) for key, value in path_section.items() if value != "no"}


def setup(config, workdir, mpi=None):
    """Run the workflow named by [workflow] mode (scripts/sprun:55-89): every
    module it lists is created from its section's ``method`` and given
    ``.config``, ``.path`` and ``.mpi`` before ``setup(workflow)``.  Returns
    the workflow after it ran."""
    paths = resolve_paths(config["path"], workdir)
    makedirs(paths["output"], exist_ok=True)
    wf = WORKFLOWS[config["workflow"]["mode"]]()
    wf.dict, wf.mpi = paths, mpi
    wf.setup()
    for section in wf.modules:
        module = load_module(section, config[section].get("method", "default"))
        module.config, module.path, module.mpi = config[section], paths, mpi
        module.setup(wf)
        setattr(wf, section, module)
    wf.run()
    return wf


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workdir", nargs="?", default=getcwd())
    ap.add_argument("--config_file", nargs="?", default="config.ini")
    args = ap.parse_args(argv)
    config, workdir = parse_config(args.workdir, args.config_file)
    if config["workflow"].get("mpi", "no") == "yes":
        from .parallel import TorchMPI
        return setup(config, workdir, TorchMPI())
    return setup(config, workdir)


if __name__ == "__main__":
    main()
