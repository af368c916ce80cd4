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


def parse_config(workdir: str, config_file: str):
    """sprun:10-42."""
    config_path = path.join(workdir, config_file)
    if not path.exists(workdir) or not path.exists(config_path):
        raise FileNotFoundError(config_path)
    config = ConfigParser()
    config.read(config_path)
    if "inherit" in config["workflow"]:
        parent_name = config["workflow"]["inherit"]
        parent, _ = parse_config(workdir + "/../" + parent_name, config_file)
        for section in ["workflow", "slurm", "preprocess", "solver", "postprocess", "optimize", "path"]:
            if section not in parent:
                continue
            if section not in config:
                config[section] = parent[section]
                if section == "path":
                    for key in config[section]:
                        if config[section][key] != "no":
                            config[section][key] = "../" + parent_name + "/" + config[section][key]
            else:
                for key in parent[section]:
                    if key not in config[section]:
                        if section == "path" and parent[section][key] != "no":
                            config[section][key] = "../" + parent_name + "/" + parent[section][key]
                        else:
                            config[section][key] = parent[section][key]
    return config, workdir


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


def setup(config, workdir, mpi=None):
    """sprun:55-89; returns the workflow after running it."""
    path_dict = {}
    for d in config["path"]:
        if config["path"][d] != "no":
            path_dict[d] = path.join(workdir, config["path"][d])
    if not path.exists(path_dict["output"]):
        makedirs(path_dict["output"])
    mode = config["workflow"]["mode"]
    wf = WORKFLOWS[mode]()
    wf.dict = path_dict
    wf.mpi = mpi
    wf.setup()
    for section in wf.modules:
        method = config[section]["method"] if "method" in config[section] else "default"
        module = load_module(section, method)
        module.config = config[section]
        module.path = path_dict
        module.mpi = mpi
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
