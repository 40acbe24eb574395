"""Exception types of the drop-in surface (same names and meaning as
util/exceptions.py:6-126 of MesoHOPS)."""


class UnsupportedRequest(Exception):
    """A request (option, parameter value) the code does not support."""

    def __init__(self, request, function, override=False):
        super().__init__(request, function)
        self.request = request
        self.function = function
        self.override = override

    def __str__(self):
        if self.override:
            return f"{self.request} in the {self.function} function."
        return (f"The current code does not support {self.request} in the "
                f"{self.function} function.")


class LockedException(Exception):
    """An operation on an object that is locked (e.g. re-initialization)."""

    def __init__(self, func_name, class_name=""):
        super().__init__(func_name)
        self.func_name = func_name
        self.class_name = class_name

    def __str__(self):
        return f"The {self.class_name} is currently locked - the attempt to access " \
               f"{self.func_name} has been canceled."


class AuxError(Exception):
    """Misconfigured auxiliary vector / hierarchy."""

    def __init__(self, sub_msg):
        super().__init__(sub_msg)
        self.sub_msg = sub_msg

    def __str__(self):
        return "There is a problem in the hierarchy: " + str(self.sub_msg)


class TrajectoryError(Exception):
    """Misconfigured or failed trajectory (time axis, noise length, NaN state)."""

    def __init__(self, sub_msg):
        super().__init__(sub_msg)
        self.sub_msg = sub_msg

    def __str__(self):
        return "There is a problem with the trajectory: " + str(self.sub_msg)
