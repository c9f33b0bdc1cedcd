"""The commands that profiles/*.md give for their captures run committed
scripts with options those scripts still accept (bench.py and
akantu_b200.train_surrogate), and every ncu command keeps the clocks
unlocked (--clock-control none)."""
import ast
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def accepted_options(path):
    """The --options of a script's argparse add_argument calls."""
    tree = ast.parse(open(path).read())
    opts = set()
    for node in ast.walk(tree):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", "") == "add_argument":
            for a in node.args:
                if isinstance(a, ast.Constant) and str(a.value).startswith("--"):
                    opts.add(a.value)
    return opts


SCRIPTS = {
    "bench.py": os.path.join(ROOT, "bench.py"),
    "akantu_b200.train_surrogate": os.path.join(ROOT, "akantu_b200", "train_surrogate.py"),
}


def commands():
    """(profile, script, options) of every command line in the profiles'
    code blocks (continuation lines joined)."""
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        for block in re.findall(r"```\n(.*?)```", open(path).read(), flags=re.S):
            text = block.replace("\\\n", " ")
            for line in text.splitlines():
                for script in SCRIPTS:
                    pattern = r"python (?:-m )?%s((?:\s+[^\s>&|;]+)*)" % re.escape(script)
                    for m in re.finditer(pattern, line):
                        yield os.path.basename(path), script, re.findall(r"(--[\w-]+)", m.group(1))


def test_profile_commands_use_accepted_options():
    found = list(commands())
    assert len(found) >= 10
    for name, script, opts in found:
        bad = set(opts) - accepted_options(SCRIPTS[script])
        assert not bad, (name, script, bad)


def test_ncu_commands_leave_clocks_alone():
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        for block in re.findall(r"```\n(.*?)```", open(path).read(), flags=re.S):
            for line in block.replace("\\\n", " ").splitlines():
                if re.search(r"(^|\s)ncu\s", line):
                    assert "--clock-control none" in line, (os.path.basename(path), line)
